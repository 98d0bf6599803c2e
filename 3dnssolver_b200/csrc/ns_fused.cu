// ns_fused.cu -- dispatch of the fused stage kernel (ns_fused.cuh) by precision
// and semantics; the kernels are compiled in ns_fused_{ref,phys}{,64}.cu.
#include "ns_fused.cuh"

namespace nsb {

cudaError_t launch_stage_fused(const FusedArgs& a, cudaStream_t s) {
    if (a.fp32) return a.phys ? fused_launch<float, true>(a, s) : fused_launch<float, false>(a, s);
    return a.phys ? fused_launch<double, true>(a, s) : fused_launch<double, false>(a, s);
}

}  // namespace nsb
