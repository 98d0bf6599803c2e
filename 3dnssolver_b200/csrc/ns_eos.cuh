// ns_eos.cuh -- equation of state, CFL time step and block reductions (device).
#pragma once

#include <cmath>

#include "ns_common.cuh"

namespace nsb {

// ---------------------------------------------------------------------------
// equation of state (src/eq_of_state.cpp:32-87)

__device__ __forceinline__ void prim_from_cons(const double u[5], double gm1, double w[5]) {
    double ir = 1.0 / u[0];
    w[0] = u[0];
    w[2] = u[2] * ir;
    w[3] = u[3] * ir;
    w[4] = u[4] * ir;
    double kin = 0.5 * (w[2] * w[2] + w[3] * w[3] + w[4] * w[4]);
    w[1] = gm1 * (u[1] - u[0] * kin);
}

__device__ __forceinline__ void cons_from_prim(const double w[5], double inv_gm1, double u[5]) {
    u[0] = w[0];
    u[2] = w[0] * w[2];
    u[3] = w[0] * w[3];
    u[4] = w[0] * w[4];
    double kin = 0.5 * w[0] * (w[2] * w[2] + w[3] * w[3] + w[4] * w[4]);
    u[1] = w[1] * inv_gm1 + kin;
}

// EqOfState::local_dt (src/eq_of_state.cpp:89-101), min over directions
__device__ __forceinline__ double local_dt(const double w[5], const Consts& c) {
    double cs = sqrt(c.gamma * w[1] / w[0]);
    double ex = c.dx / fmax(fabs(w[2] + cs), fabs(w[2] - cs));
    double ey = c.dy / fmax(fabs(w[3] + cs), fabs(w[3] - cs));
    double ez = c.dz / fmax(fabs(w[4] + cs), fabs(w[4] - cs));
    double t = (ey < ex) ? ey : ex;
    return (ez < t) ? ez : t;
}

__device__ __forceinline__ double local_dt_physical(const double w[5], const Consts& c) {
    double cs = sqrt(c.gamma * w[1] / w[0]);
    double r = (fabs(w[2]) + cs) * c.inv_dx + (fabs(w[3]) + cs) * c.inv_dy;
    if (c.dim == 3) r += (fabs(w[4]) + cs) * c.inv_dz;
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
