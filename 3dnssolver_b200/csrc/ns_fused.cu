// ns_fused.cu -- dispatch of the fused FP32 stage kernel (ns_fused.cuh) by
// semantics; the kernels are compiled in ns_fused_ref.cu and ns_fused_phys.cu.
#include "ns_fused.cuh"

namespace nsb {

cudaError_t launch_stage_fused(const FusedArgs& a, cudaStream_t s) {
    if (!a.fp32) return cudaErrorInvalidValue;
    return a.phys ? fused_launch<float, true>(a, s) : fused_launch<float, false>(a, s);
}

}  // namespace nsb
