// ns_fused_phys.cu -- the fused FP32 stage kernels of the physical semantics.
#include "ns_fused.cuh"

namespace nsb {
template cudaError_t fused_launch<float, true>(const FusedArgs& a, cudaStream_t s);
}  // namespace nsb
