// ns_fused_phys64.cu -- the fused FP64 stage kernels of the physical semantics.
#include "ns_fused.cuh"

namespace nsb {
template cudaError_t fused_launch<double, true>(const FusedArgs& a, cudaStream_t s);
}  // namespace nsb
