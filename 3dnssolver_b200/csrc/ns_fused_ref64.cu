// ns_fused_ref64.cu -- the fused FP64 stage kernels of the reference semantics.
#include "ns_fused.cuh"

namespace nsb {
template cudaError_t fused_launch<double, false>(const FusedArgs& a, cudaStream_t s);
}  // namespace nsb
