// ns_fused_ref.cu -- the fused FP32 stage kernels of the reference semantics.
#include "ns_fused.cuh"

namespace nsb {
template cudaError_t fused_launch<float, false>(const FusedArgs& a, cudaStream_t s);
}  // namespace nsb
