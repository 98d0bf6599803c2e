// ns_gate.cu -- the learned sensor's correction of a fused FP32 stage (no
// reference counterpart).
//
// A sensor-gated time step runs the component-wise fused stage kernel on every
// face (ns_fused.cuh) and then corrects the faces the sensor flagged:
//   k_gate_delta  one thread per flagged face (a compacted list per axis): the
//                 characteristic-wise minus the component-wise flux of that face,
//                 from the stage's input state, into the face array of its axis
//                 (Weno5cw::compute_num_flux vs Weno5::*_sweep,
//                 src/convection_schemes/weno-5cw.cpp:4-28, weno-5.cpp:96-114)
//   k_gate_apply  one thread per cell next to a flagged face (a compacted list):
//                 U_out += mc dt sum_axes (d(+) - d(-)) / dx_axis over its flagged
//                 faces, in the fixed order of the residual (Weno5::compute_residual,
//                 weno-5.cpp:39-73); in the third stage also the next step's start
//                 of those cells (the fused kernel leaves it to this pass).
// Each flagged face is evaluated once per stage, the sums run in a fixed order
// (no atomics on the state), and a step whose sensor fires nowhere costs the
// component-wise stages plus six launches that find empty lists.
#include <cuda_runtime.h>

#include "ns_common.cuh"
#include "ns_eos.cuh"
#include "ns_face.cuh"
#include "ns_face_f32x2.cuh"
#include "ns_kernels.h"
#include "ns_sensor.h"

namespace nsb {

constexpr int GT = 128;  // threads per block of the correction kernels

// W = prim(U) in FP32 arithmetic from the FP64 state, as the fused stage kernel
// forms its plane ring (ns_fused.cuh convert_plane), so that the component-wise
// flux formed here is the one the stage used
__device__ __forceinline__ void w32_from_u(const double* __restrict__ U, long long fs, long long o, float gm1,
                                           float w[5]) {
    float u[5];
#pragma unroll
    for (int q = 0; q < 5; q++) u[q] = float(U[q * fs + o]);
    const float ir = __fdividef(1.f, u[0]);
    const float vx = u[2] * ir, vy = u[3] * ir, vz = u[4] * ir;
    w[0] = u[0];
    w[1] = gm1 * (u[1] - 0.5f * u[0] * (vx * vx + vy * vy + vz * vz));
    w[2] = vx;
    w[3] = vy;
    w[4] = vz;
}

template <int DIR, bool BORGES, bool PHYS>
__global__ void __launch_bounds__(GT) k_gate_delta(const double* __restrict__ Uin, Box b, Consts c,
                                                   const unsigned* __restrict__ list,
                                                   const unsigned* __restrict__ count, FaceBox fb,
                                                   float* __restrict__ D) {
    // the stencil's W of every thread, [q][s][thread]: face_f32x2 reads cell s of
    // component q at q * (6 GT) + s * GT + thread
    __shared__ float ws[5 * 6 * GT];
    const unsigned n = *count;
    const float gamma = float(c.gamma), inv_gm1 = float(c.inv_gm1), gm1 = float(c.gm1);
    const float* planes[6] = {ws, ws, ws, ws, ws, ws};
    for (unsigned e = blockIdx.x * GT + threadIdx.x; e < n; e += gridDim.x * GT) {
        const unsigned f = list[e];
        const int kk = (int)(f % (unsigned)fb.n2), bb = (int)((f / (unsigned)fb.n2) % (unsigned)fb.n1),
                  aa = (int)(f / ((unsigned)fb.n2 * (unsigned)fb.n1));
        // face aa (along DIR) lies between cells aa-1 and aa: stencil aa-3 .. aa+2
#pragma unroll
        for (int s = 0; s < 6; s++) {
            int i = aa, j = bb, k = kk;
            if (DIR == 0) i = fold(aa - 3 + s, b.nx, c.periodic[0]);
            if (DIR == 1) j = fold(bb - 3 + s, b.ny, c.periodic[1]);
            if (DIR == 2) k = fold(kk - 3 + s, b.nz, c.periodic[2]);
            float w[5];
            w32_from_u(Uin, b.fstride, b.at(i + NG, j + NG, k + NG), gm1, w);
#pragma unroll
            for (int q = 0; q < 5; q++) ws[(q * 6 + s) * GT + threadIdx.x] = w[q];
        }
        float fc[5], fx[5];
        face_f32x2<DIR, false, BORGES, PHYS>(planes, threadIdx.x, GT, 6 * GT, gamma, inv_gm1, fc);
        face_f32x2<DIR, true, BORGES, PHYS>(planes, threadIdx.x, GT, 6 * GT, gamma, inv_gm1, fx);
#pragma unroll
        for (int q = 0; q < 5; q++) D[q * fb.fstride + f] = fx[q] - fc[q];
    }
}

template <bool LAST, bool PHYS>
__global__ void __launch_bounds__(GT) k_gate_apply(const unsigned* __restrict__ cells,
                                                   const unsigned* __restrict__ count, Gate g,
                                                   const float* __restrict__ D0, const float* __restrict__ D1,
                                                   const float* __restrict__ D2, Box b, Consts c, int conv_dims,
                                                   double mc, double* __restrict__ Uout, double* __restrict__ U0,
                                                   const unsigned long long* __restrict__ slot,
                                                   unsigned long long* __restrict__ slot_next) {
    const unsigned n = *count;
    const double m3 = mc * fmin(1e10, __longlong_as_double((long long)*slot)) * c.cfl;
    const double inv[3] = {c.inv_dx, c.inv_dy, c.inv_dz};
    const float* D[3] = {D0, D1, D2};
    double best = INFINITY;
    for (unsigned e = blockIdx.x * GT + threadIdx.x; e < n; e += gridDim.x * GT) {
        const unsigned cell = cells[e];
        const int k = (int)(cell % (unsigned)b.nz), j = (int)((cell / (unsigned)b.nz) % (unsigned)b.ny),
                  i = (int)(cell / ((unsigned)b.nz * (unsigned)b.ny));
        double r[5] = {0, 0, 0, 0, 0};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (d >= conv_dims) break;
            const FaceBox& fb = g.fb[d];
            // the faces below and above the cell along d (face f lies between cells f-1 and f)
            const long long fm = fb.at(i, j, k);
            const long long fp = d == 0 ? fb.at(i + 1, j, k) : (d == 1 ? fb.at(i, j + 1, k) : fb.at(i, j, k + 1));
            const bool am = g.m[d][fm] != 0, ap = g.m[d][fp] != 0;
#pragma unroll
            for (int q = 0; q < 5; q++) {
                const double dp = ap ? double(D[d][q * fb.fstride + fp]) : 0.0;
                const double dm = am ? double(D[d][q * fb.fstride + fm]) : 0.0;
                r[q] += (dp - dm) * inv[d];
            }
        }
        const long long o = b.at(i + NG, j + NG, k + NG);
        double un[5];
#pragma unroll
        for (int q = 0; q < 5; q++) {
            un[q] = Uout[q * b.fstride + o] + r[q] * m3;
            Uout[q * b.fstride + o] = un[q];
        }
        if constexpr (LAST) {  // the next step's start of this cell (the fused kernel skipped it)
            double w[5], u0[5];
            prim_from_cons(un, c.gm1, w);
            const double dd = PHYS ? local_dt_physical(w, c) : local_dt(w, c);
            if (dd < best) best = dd;
            cons_from_prim(w, c.inv_gm1, u0);
#pragma unroll
            for (int q = 0; q < 5; q++) U0[q * b.fstride + o] = u0[q];
        }
    }
    if constexpr (LAST) block_min_to(best, slot_next);
}

template <int DIR, bool PHYS>
static void delta_one(bool borges, const FusedArgs& a, const GateLists& L, void* F, const FaceBox& fb, int grid,
                      cudaStream_t s) {
    if (borges)
        k_gate_delta<DIR, true, PHYS><<<grid, GT, 0, s>>>(a.Uin, a.b, a.c, L.face_list[DIR], L.face_count + DIR, fb,
                                                          (float*)F);
    else
        k_gate_delta<DIR, false, PHYS><<<grid, GT, 0, s>>>(a.Uin, a.b, a.c, L.face_list[DIR], L.face_count + DIR,
                                                           fb, (float*)F);
}

// Persistent grids sized for full residency: the delta kernel (100 registers)
// fits 5 blocks per SM, the apply kernel (32 registers) 16; both are bound by
// the latency of their scattered loads, so every resident warp counts.
template <bool PHYS>
static void gate_correct_t(const FusedArgs& a, const GateLists& L, void* const F[3], const FaceBox fb[3], int sms,
                           cudaStream_t s) {
    const int grid_delta = sms * 5, grid = sms * 16;
    for (int d = 0; d < a.conv_dims; d++) {
        if (d == 0) delta_one<0, PHYS>(a.borges, a, L, F[0], fb[0], grid_delta, s);
        else if (d == 1) delta_one<1, PHYS>(a.borges, a, L, F[1], fb[1], grid_delta, s);
        else delta_one<2, PHYS>(a.borges, a, L, F[2], fb[2], grid_delta, s);
    }
    Gate g;
    for (int d = 0; d < 3; d++) { g.m[d] = L.mask[d]; g.fb[d] = fb[d]; }
    if (a.last)
        k_gate_apply<true, PHYS><<<grid, GT, 0, s>>>(L.cell_list, L.cell_count, g, (const float*)F[0],
                                                     (const float*)F[1], (const float*)F[2], a.b, a.c, a.conv_dims,
                                                     a.mc, a.Uout, a.U0, a.slot, a.slot_next);
    else
        k_gate_apply<false, PHYS><<<grid, GT, 0, s>>>(L.cell_list, L.cell_count, g, (const float*)F[0],
                                                      (const float*)F[1], (const float*)F[2], a.b, a.c, a.conv_dims,
                                                      a.mc, a.Uout, a.U0, a.slot, a.slot_next);
}

cudaError_t gate_correct(const FusedArgs& a, const GateLists& L, void* const F[3], const FaceBox fb[3], int sms,
                         cudaStream_t s) {
    // persistent: the list lengths stay on the device
    if (a.phys) gate_correct_t<true>(a, L, F, fb, sms, s);
    else gate_correct_t<false>(a, L, F, fb, sms, s);
    return cudaGetLastError();
}

}  // namespace nsb
