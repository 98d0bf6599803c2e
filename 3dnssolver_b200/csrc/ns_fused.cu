// ns_fused.cu -- one kernel per SSP-RK3 stage (reference semantics).
//
// A block owns a TX x TY x TZ tile of interior cells.  It loads the tile's box
// with 3 ghost layers on every side once, folding each axis by its boundary
// condition (periodic wrap or Neumann clamp: the single-GPU form of
// Domain::apply_boundary_conditions + Communicator::communicate,
// src/domain.cpp:18-28, src/communicator.cpp:6-143), and keeps W = prim(U)
// (src/eq_of_state.cpp:61-87) in shared memory.  From there it computes the
// face fluxes of the tile along x, then y, then z into a shared face buffer,
// accumulating each cell's (f(+) - f(-))/d in the reference's order
// (Weno5::compute_residual, weno-5.cpp:39-73), adds the centered viscous terms
// from the same box, and writes U_out = U0 m1 + U_in m2 + R mc dt
// (TimeScheme::substep, time_scheme.cpp:72-96).  U_in and U_out are different
// buffers: neighbouring blocks read U_in's cells as their ghost layers.
//
// The third stage also takes the next step's start: W = prim(U_out) for the
// CFL minimum (time_scheme.cpp:69, 98-136) and U0 = cons(W) (the W -> U
// round trip of time_scheme.cpp:124), so a step is three launches.
//
// The Lax-Friedrichs split uses U = cons(W) of the boxed W; it differs from
// the stage's U by rounding only.
#include <cuda_runtime.h>

#include "ns_common.cuh"
#include "ns_eos.cuh"
#include "ns_face.cuh"
#include "ns_kernels.h"
#include "ns_viscous.cuh"

namespace nsb {

constexpr int FT = 256;  // threads per block

template <typename T>
struct Tile {
    static constexpr int TX = 4, TY = 4, TZ = 32;  // 512 cells, 2 per thread
    static constexpr int BX = TX + 6, BY = TY + 6, BZ = TZ + 6;
    static constexpr int NB = BX * BY * BZ;  // boxed cells
    static constexpr int NF = (TX + 1) * TY * TZ > TX * TY * (TZ + 1) ? (TX + 1) * TY * TZ
                                                                      : TX * TY * (TZ + 1);
    static constexpr int NC = TX * TY * TZ;
    static constexpr int MINB = sizeof(T) == 8 ? 1 : 2;
    static constexpr size_t smem = (size_t)5 * NB * sizeof(T) + (size_t)5 * NF * sizeof(T) +
                                   (size_t)5 * NC * sizeof(double);
};

// faces of the tile along DIR into Fs, then r += (f(+) - f(-)) / d for the owned cells
template <int DIR, bool CHAR, bool BORGES, typename T>
__device__ __forceinline__ void fused_face_pass(const T* __restrict__ Ws, T* __restrict__ Fs,
                                                double* __restrict__ Rs, T gamma, T inv_gm1,
                                                double inv_d) {
    using G = Tile<T>;
    constexpr int FA = G::TX + (DIR == 0), FB = G::TY + (DIR == 1), FC = G::TZ + (DIR == 2);
    constexpr int NFD = FA * FB * FC;
    constexpr int step = DIR == 0 ? G::BY * G::BZ : (DIR == 1 ? G::BZ : 1);
    const T hg = T(0.5) * gamma * inv_gm1;
    for (int e = threadIdx.x; e < NFD; e += FT) {
        int fc = e % FC, t = e / FC, fb = t % FB, fa = t / FB;
        // stencil cell 0 of face f along DIR is tile cell f-3, box coordinate f
        int bx = fa + (DIR == 0 ? 0 : 3), by = fb + (DIR == 1 ? 0 : 3), bz = fc + (DIR == 2 ? 0 : 3);
        int base = (bx * G::BY + by) * G::BZ + bz;
        T fL[5][5], fR[5][5], wa[5], out[5];
#pragma unroll
        for (int s = 0; s < 6; s++) {
            int idx = base + s * step;
            T w[5], u[5];
#pragma unroll
            for (int q = 0; q < 5; q++) w[q] = Ws[q * G::NB + idx];
            // U = cons(W) (eq_of_state.cpp:32-59)
            u[0] = w[0];
            u[2] = w[0] * w[2];
            u[3] = w[0] * w[3];
            u[4] = w[0] * w[4];
            u[1] = w[1] * inv_gm1 + T(0.5) * w[0] * (w[2] * w[2] + w[3] * w[3] + w[4] * w[4]);
            split_cell<DIR, CHAR, T>(s, w, u, hg, fL, fR, wa);
        }
        if constexpr (CHAR)
            face_char<DIR, false, T, BORGES>(fL, fR, wa, gamma, inv_gm1, out);
        else
            face_comp<T, BORGES>(fL, fR, out);
#pragma unroll
        for (int q = 0; q < 5; q++) Fs[q * G::NF + e] = out[q];
    }
    __syncthreads();
    for (int cidx = threadIdx.x; cidx < G::NC; cidx += FT) {
        int lk = cidx % G::TZ, t = cidx / G::TZ, lj = t % G::TY, li = t / G::TY;
        int left = (li * FB + lj) * FC + lk;
        int right = left + (DIR == 0 ? FB * FC : (DIR == 1 ? FC : 1));
#pragma unroll
        for (int q = 0; q < 5; q++)
            Rs[q * G::NC + cidx] += (double(Fs[q * G::NF + right]) - double(Fs[q * G::NF + left])) * inv_d;
    }
    __syncthreads();
}

// centered viscous terms of tile cell (li, lj, lk) from the box (reference semantics):
// mixed derivatives differentiate first derivatives that are zero outside the
// interior along a non-periodic axis (centered_diffusion.cpp:22-24)
template <int H, typename T>
__device__ __forceinline__ void fused_viscous(const T* __restrict__ Ws, const Consts& c, int nx,
                                              int ny, int gi, int gj, int li, int lj, int lk,
                                              T r[5]) {
    using G = Tile<T>;
    const int sx = G::BY * G::BZ, sy = G::BZ;
    const int o = ((li + 3) * G::BY + (lj + 3)) * G::BZ + (lk + 3);
    T cx1[2 * H + 1], cy1[2 * H + 1], cxx[2 * H + 1], cyy[2 * H + 1];
#pragma unroll
    for (int t = 0; t <= 2 * H; t++) {
        cx1[t] = T(c.df[3 - H + t] * c.inv_dx);
        cy1[t] = T(c.df[3 - H + t] * c.inv_dy);
        cxx[t] = T(c.ddf[3 - H + t] * c.inv_dx * c.inv_dx);
        cyy[t] = T(c.ddf[3 - H + t] * c.inv_dy * c.inv_dy);
    }
    T Dx[4], Dy[4], Dxx[4], Dyy[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        T a1 = 0, b1 = 0, a2 = 0, b2 = 0;
#pragma unroll
        for (int t = 0; t <= 2 * H; t++) {
            T wx = Ws[q * G::NB + o + (t - H) * sx];
            T wy = Ws[q * G::NB + o + (t - H) * sy];
            if (t != H) { a1 += wx * cx1[t]; b1 += wy * cy1[t]; }
            a2 += wx * cxx[t];
            b2 += wx * cyy[t];  // d2/dy2 uses the x-stencil (cd-n.cpp:77)
        }
        Dx[q] = a1; Dy[q] = b1; Dxx[q] = a2; Dyy[q] = b2;
    }
    T Dxy[2], Dyx[2];
#pragma unroll
    for (int v = 0; v < 2; v++) {
        const int q = 2 + v;
        T sxy = 0, syx = 0;
#pragma unroll
        for (int s = 0; s <= 2 * H; s++) {
            if (s == H) continue;
            int jj = gj + s - H;
            if ((jj >= 0 && jj < ny) || c.periodic[1]) {
                T dx = 0;
#pragma unroll
                for (int t = 0; t <= 2 * H; t++)
                    if (t != H) dx += Ws[q * G::NB + o + (s - H) * sy + (t - H) * sx] * cx1[t];
                sxy += dx * cy1[s];
            }
            int ii = gi + s - H;
            if ((ii >= 0 && ii < nx) || c.periodic[0]) {
                T dy = 0;
#pragma unroll
                for (int t = 0; t <= 2 * H; t++)
                    if (t != H) dy += Ws[q * G::NB + o + (s - H) * sx + (t - H) * sy] * cy1[t];
                syx += dy * cx1[s];
            }
        }
        Dxy[v] = sxy; Dyx[v] = syx;
    }
    viscous_reference_terms<T>(Dx, Dy, Dxx, Dyy, Dxy, Dyx, Ws[2 * G::NB + o], Ws[3 * G::NB + o],
                               Ws[1 * G::NB + o], Ws[o], c, r);
}

template <typename T, bool CHAR, bool BORGES, int H, bool LAST>
__global__ void __launch_bounds__(FT, Tile<T>::MINB)
    k_stage_fused(const double* __restrict__ Uin, double* U0, double* __restrict__ Uout, Box b,
                  Consts c, int conv_dims, double m1, double m2, double mc,
                  const unsigned long long* __restrict__ slot, unsigned long long* slot_next,
                  double* clock) {
    using G = Tile<T>;
    extern __shared__ __align__(16) unsigned char smem[];
    T* Ws = reinterpret_cast<T*>(smem);
    T* Fs = Ws + 5 * G::NB;
    double* Rs = reinterpret_cast<double*>(Fs + 5 * G::NF);
    const int i0 = blockIdx.z * G::TX, j0 = blockIdx.y * G::TY, k0 = blockIdx.x * G::TZ;
    // 1. box of W = prim(U_in) at folded positions
    for (int e = threadIdx.x; e < G::NB; e += FT) {
        int bz = e % G::BZ, t = e / G::BZ, by = t % G::BY, bx = t / G::BY;
        int gi = fold(i0 - 3 + bx, b.nx, c.periodic[0]);
        int gj = fold(j0 - 3 + by, b.ny, c.periodic[1]);
        int gk = fold(k0 - 3 + bz, b.nz, c.periodic[2]);
        long long o = b.at(gi + NG, gj + NG, gk + NG);
        double u[5], w[5];
#pragma unroll
        for (int q = 0; q < 5; q++) u[q] = Uin[q * b.fstride + o];
        prim_from_cons(u, c.gm1, w);
#pragma unroll
        for (int q = 0; q < 5; q++) Ws[q * G::NB + e] = T(w[q]);
    }
    for (int e = threadIdx.x; e < 5 * G::NC; e += FT) Rs[e] = 0.0;
    __syncthreads();
    // 2. convective residual, x then y then z
    const T gamma = T(c.gamma), inv_gm1 = T(c.inv_gm1);
    if (conv_dims > 0) {
        fused_face_pass<0, CHAR, BORGES, T>(Ws, Fs, Rs, gamma, inv_gm1, c.inv_dx);
        fused_face_pass<1, CHAR, BORGES, T>(Ws, Fs, Rs, gamma, inv_gm1, c.inv_dy);
        if (conv_dims == 3) fused_face_pass<2, CHAR, BORGES, T>(Ws, Fs, Rs, gamma, inv_gm1, c.inv_dz);
    }
    // 3. viscous terms + RK combination for the owned cells
    const double dt = fmin(1e10, __longlong_as_double((long long)*slot)) * c.cfl;
    const double m3 = mc * dt;
    if (clock && (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x) == 0) {
        clock[0] = dt;
        clock[1] += dt;
    }
    double best = INFINITY;
    for (int cidx = threadIdx.x; cidx < G::NC; cidx += FT) {
        int lk = cidx % G::TZ, t = cidx / G::TZ, lj = t % G::TY, li = t / G::TY;
        int gi = i0 + li, gj = j0 + lj, gk = k0 + lk;
        if (gi >= b.nx || gj >= b.ny || gk >= b.nz) continue;
        double r[5];
#pragma unroll
        for (int q = 0; q < 5; q++) r[q] = Rs[q * G::NC + cidx];
        if constexpr (H > 0) {
            T rv[5] = {0, 0, 0, 0, 0};
            fused_viscous<H, T>(Ws, c, b.nx, b.ny, gi, gj, li, lj, lk, rv);
#pragma unroll
            for (int q = 1; q < 5; q++) r[q] += double(rv[q]);
        }
        long long o = b.at(gi + NG, gj + NG, gk + NG);
        double un[5];
#pragma unroll
        for (int q = 0; q < 5; q++) {
            long long a = q * b.fstride + o;
            un[q] = (U0[a] * m1) + (Uin[a] * m2) + (r[q] * m3);
            Uout[a] = un[q];
        }
        if constexpr (LAST) {
            // start of the next step: W = prim(U), its CFL minimum, U0 = cons(W)
            double w[5], u0[5];
            prim_from_cons(un, c.gm1, w);
            double d = local_dt(w, c);
            if (d < best) best = d;
            cons_from_prim(w, c.inv_gm1, u0);
#pragma unroll
            for (int q = 0; q < 5; q++) U0[q * b.fstride + o] = u0[q];
        }
    }
    if constexpr (LAST) block_min_to(best, slot_next);
}

template <typename T, bool CHAR, bool BORGES, int H, bool LAST>
static cudaError_t fused_one(const FusedArgs& a, cudaStream_t s) {
    using G = Tile<T>;
    auto kern = k_stage_fused<T, CHAR, BORGES, H, LAST>;
    // the attribute is per device; setting it on every launch keeps multi-device use correct
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem);
    if (e != cudaSuccess) return e;
    dim3 grid((a.b.nz + G::TZ - 1) / G::TZ, (a.b.ny + G::TY - 1) / G::TY, (a.b.nx + G::TX - 1) / G::TX);
    kern<<<grid, FT, G::smem, s>>>(a.Uin, a.U0, a.Uout, a.b, a.c, a.conv_dims, a.m1, a.m2, a.mc, a.slot,
                                   a.slot_next, a.clock);
    return cudaGetLastError();
}

template <typename T, bool CHAR, bool BORGES, bool LAST>
static cudaError_t fused_h(const FusedArgs& a, cudaStream_t s) {
    switch (a.visc_h) {
        case 0: return fused_one<T, CHAR, BORGES, 0, LAST>(a, s);
        case 1: return fused_one<T, CHAR, BORGES, 1, LAST>(a, s);
        case 2: return fused_one<T, CHAR, BORGES, 2, LAST>(a, s);
        default: return fused_one<T, CHAR, BORGES, 3, LAST>(a, s);
    }
}

template <typename T>
static cudaError_t fused_t(const FusedArgs& a, cudaStream_t s) {
    if (a.chr) {
        if (a.borges) return a.last ? fused_h<T, true, true, true>(a, s) : fused_h<T, true, true, false>(a, s);
        return a.last ? fused_h<T, true, false, true>(a, s) : fused_h<T, true, false, false>(a, s);
    }
    if (a.borges) return a.last ? fused_h<T, false, true, true>(a, s) : fused_h<T, false, true, false>(a, s);
    return a.last ? fused_h<T, false, false, true>(a, s) : fused_h<T, false, false, false>(a, s);
}

cudaError_t launch_stage_fused(const FusedArgs& a, cudaStream_t s) {
    return a.fp32 ? fused_t<float>(a, s) : fused_t<double>(a, s);
}

}  // namespace nsb
