// ns_eos.cuh -- equation of state, CFL time step and block reductions (device).
#pragma once

#include <cmath>

#include "ns_common.cuh"

namespace nsb {

// ---------------------------------------------------------------------------
// equation of state (src/eq_of_state.cpp:32-87)

// The roundings are written out (__dmul_rn / __fma_rn) so that every kernel that
// inlines these forms the same bits: the step start formed inside a stage kernel
// then equals the one a separate kernel forms from a downloaded W, and a restart
// from written fields reproduces an uninterrupted run exactly.
__device__ __forceinline__ double sum_sq3(double a, double b, double c) {
    return __fma_rn(c, c, __fma_rn(b, b, __dmul_rn(a, a)));
}

__device__ __forceinline__ void prim_from_cons(const double u[5], double gm1, double w[5]) {
    double ir = 1.0 / u[0];
    w[0] = u[0];
    w[2] = __dmul_rn(u[2], ir);
    w[3] = __dmul_rn(u[3], ir);
    w[4] = __dmul_rn(u[4], ir);
    double kin = __dmul_rn(0.5, sum_sq3(w[2], w[3], w[4]));
    w[1] = __dmul_rn(gm1, __fma_rn(-u[0], kin, u[1]));
}

__device__ __forceinline__ void cons_from_prim(const double w[5], double inv_gm1, double u[5]) {
    u[0] = w[0];
    u[2] = __dmul_rn(w[0], w[2]);
    u[3] = __dmul_rn(w[0], w[3]);
    u[4] = __dmul_rn(w[0], w[4]);
    double kin = __dmul_rn(__dmul_rn(0.5, w[0]), sum_sq3(w[2], w[3], w[4]));
    u[1] = __fma_rn(w[1], inv_gm1, kin);
}

// EqOfState::local_dt (src/eq_of_state.cpp:89-101), min over directions
// max(|u+c|, |u-c|) is |u| + c for c >= 0, exactly and in rounding; the minimum
// over the axes of d/(|u|+c) is taken as one reciprocal of the largest (|u|+c)/d
// (within 2 ulp of the reference's three divisions; NaN still yields NaN)
__device__ __forceinline__ double local_dt(const double w[5], const Consts& c) {
    double cs = sqrt(c.gamma * w[1] / w[0]);
    double rx = __dmul_rn(fabs(w[2]) + cs, c.inv_dx);
    double ry = __dmul_rn(fabs(w[3]) + cs, c.inv_dy);
    double rz = __dmul_rn(fabs(w[4]) + cs, c.inv_dz);
    return 1.0 / fmax(rx, fmax(ry, rz));
}

__device__ __forceinline__ double local_dt_physical(const double w[5], const Consts& c) {
    double cs = sqrt(c.gamma * w[1] / w[0]);
    double r = __fma_rn(fabs(w[3]) + cs, c.inv_dy, __dmul_rn(fabs(w[2]) + cs, c.inv_dx));
    if (c.dim == 3) r = __fma_rn(fabs(w[4]) + cs, c.inv_dz, r);
    return 1.0 / r;
}

// block-wide min of a positive double, then one 64-bit atomicMin on its bit
// pattern (positive IEEE doubles order like their unsigned bit patterns)
__device__ __forceinline__ void block_min_to(double v, unsigned long long* slot) {
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    int lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31;
    int warp = (threadIdx.x + threadIdx.y * blockDim.x) >> 5;
    int nw = (blockDim.x * blockDim.y + 31) >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < nw ? red[lane] : INFINITY;
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0 && v < INFINITY)
            atomicMin(slot, (unsigned long long)__double_as_longlong(v));
    }
}

}  // namespace nsb
