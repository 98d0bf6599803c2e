// ns_kernels.cu -- device kernels of the explicit RHS and SSP-RK3 stage.
//
// Per RK stage (TimeScheme::step, src/time_scheme.cpp:33-66):
//   k_fill_prim      boundary fill + halo exchange of U on the face halos, then
//                    W = prim(U) on every cell (time_scheme.cpp:133-135)
//   k_face_flux<d>   WENO-5 face fluxes along axis d, one thread per face
//                    (Weno5::x/y/z_sweep, Weno5cw::*_sweep); the FP64 steps of
//                    the physical semantics run k_face_flux_tma (ns_tma.cu)
//                    for y and z and k_viscous_tma for CD-2 viscous terms
//   k_update         flux differences + centered viscous terms + RK combination
//                    (Weno5::compute_residual, CenteredDiffusion::compute_residual,
//                    TimeScheme::substep)
// Per step: k_step_begin (dt reduction over W, then U = cons(W), U0 = U).
#include <cuda_runtime.h>

#include <algorithm>

#include <cfloat>
#include <cmath>

#include "ns_common.cuh"
#include "ns_eos.cuh"
#include "ns_face.cuh"
#include "ns_kernels.h"
#include "ns_tcgen05.cuh"
#include "ns_tma.cuh"
#include "ns_viscous.cuh"

namespace nsb {

// ---------------------------------------------------------------------------
// step begin: dt from W at the step start (TimeScheme::set_dt), then
// U = cons(W) on every cell (time_scheme.cpp:124) and U0 = U (:126), also on
// every cell.
// FROM_U: the state is U after the previous step; W = prim(U) first
// (time_scheme.cpp:69).  Grid: (ceil(NZp/32), ceil(NY/4), NX).

template <bool FROM_U, bool PHYS>
__global__ void __launch_bounds__(128) k_step_begin(double* __restrict__ W, double* __restrict__ U,
                                                    double* __restrict__ U0, Box b, Consts c,
                                                    unsigned long long* __restrict__ slot, int ih0) {
    int kh = blockIdx.x * 32 + threadIdx.x;
    int jh = blockIdx.y * 4 + threadIdx.y;
    int ih = blockIdx.z + ih0;
    double best = INFINITY;
    if (kh < b.nz + 2 * NG && jh < b.NY) {
        long long o = b.at(ih, jh, kh);
        double w[5], u[5];
        if (FROM_U) {
#pragma unroll
            for (int q = 0; q < 5; q++) u[q] = U[q * b.fstride + o];
            prim_from_cons(u, c.gm1, w);
#pragma unroll
            for (int q = 0; q < 5; q++) W[q * b.fstride + o] = w[q];
        } else {
#pragma unroll
            for (int q = 0; q < 5; q++) w[q] = W[q * b.fstride + o];
        }
        bool interior = ih >= NG && ih < b.nx + NG && jh >= NG && jh < b.ny + NG && kh >= NG &&
                        kh < b.nz + NG;
        if (interior) {
            double dt = PHYS ? local_dt_physical(w, c) : local_dt(w, c);
            if (dt < best) best = dt;  // NaN never lowers the minimum (time_scheme.cpp:117)
        }
        cons_from_prim(w, c.inv_gm1, u);
#pragma unroll
        for (int q = 0; q < 5; q++) {
            U[q * b.fstride + o] = u[q];
            U0[q * b.fstride + o] = u[q];  // all cells: the stages that start from U0 keep its edges
        }
    }
    block_min_to(best, slot);
}

// W = prim(U) on every cell (end of TimeScheme::step, time_scheme.cpp:69)
__global__ void __launch_bounds__(128) k_prim_all(double* __restrict__ W, const double* __restrict__ U,
                                                  Box b, Consts c, int ih0) {
    int kh = blockIdx.x * 32 + threadIdx.x;
    int jh = blockIdx.y * 4 + threadIdx.y;
    int ih = blockIdx.z + ih0;
    if (kh >= b.nz + 2 * NG || jh >= b.NY) return;
    long long o = b.at(ih, jh, kh);
    double u[5], w[5];
#pragma unroll
    for (int q = 0; q < 5; q++) u[q] = U[q * b.fstride + o];
    prim_from_cons(u, c.gm1, w);
#pragma unroll
    for (int q = 0; q < 5; q++) W[q * b.fstride + o] = w[q];
}

// U = cons(W) on every cell
__global__ void __launch_bounds__(128) k_cons_all(const double* __restrict__ W, double* __restrict__ U,
                                                  Box b, Consts c) {
    int kh = blockIdx.x * 32 + threadIdx.x;
    int jh = blockIdx.y * 4 + threadIdx.y;
    int ih = blockIdx.z;
    if (kh >= b.nz + 2 * NG || jh >= b.NY) return;
    long long o = b.at(ih, jh, kh);
    double u[5], w[5];
#pragma unroll
    for (int q = 0; q < 5; q++) w[q] = W[q * b.fstride + o];
    cons_from_prim(w, c.inv_gm1, u);
#pragma unroll
    for (int q = 0; q < 5; q++) U[q * b.fstride + o] = u[q];
}

// CFL minimum over the interior of W (TimeScheme::get_local_max_dt, time_scheme.cpp:98-125)
template <bool PHYS>
__global__ void __launch_bounds__(128) k_min_dt(const double* __restrict__ W, Box b, Consts c,
                                                unsigned long long* __restrict__ slot) {
    int k = blockIdx.x * 32 + threadIdx.x;
    int j = blockIdx.y * 4 + threadIdx.y;
    int i = blockIdx.z;
    double best = INFINITY;
    if (k < b.nz && j < b.ny) {
        long long o = b.at(i + NG, j + NG, k + NG);
        double w[5];
#pragma unroll
        for (int q = 0; q < 5; q++) w[q] = W[q * b.fstride + o];
        double dt = PHYS ? local_dt_physical(w, c) : local_dt(w, c);
        if (dt < best) best = dt;
    }
    block_min_to(best, slot);
}

// ---------------------------------------------------------------------------
// stage prologue: Neumann copy / periodic wrap of U on the face halos
// (boundary_neumann.cpp:22-132, communicator.cpp:6-143: face regions only),
// then W = prim(U) on every cell (eq_of_state.cpp:61-87).

__global__ void __launch_bounds__(128) k_fill_prim(double* __restrict__ W, double* __restrict__ U,
                                                   Box b, Consts c, double* __restrict__ Uhalo, int ih0) {
    int kh = blockIdx.x * 32 + threadIdx.x;
    int jh = blockIdx.y * 4 + threadIdx.y;
    int ih = blockIdx.z + ih0;
    if (kh >= b.nz + 2 * NG || jh >= b.NY) return;
    int i = ih - NG, j = jh - NG, k = kh - NG;
    bool ox = i < 0 || i >= b.nx, oy = j < 0 || j >= b.ny, oz = k < 0 || k >= b.nz;
    // a slab's exchanged x ghost plane holds a neighbour's cells: its y and z ghost
    // rows fold within the plane like those of an interior plane
    if (ox && x_exchanged(i >= b.nx, b.nx, c)) ox = false;
    long long o = b.at(ih, jh, kh);
    double u[5], w[5];
    if ((int)ox + (int)oy + (int)oz == 1) {
        int si = ox ? fold(i, b.nx, c.periodic[0]) : i;
        int sj = oy ? fold(j, b.ny, c.periodic[1]) : j;
        int sk = oz ? fold(k, b.nz, c.periodic[2]) : k;
        long long s = b.at(si + NG, sj + NG, sk + NG);
#pragma unroll
        for (int q = 0; q < 5; q++) {
            u[q] = U[q * b.fstride + s];
            U[q * b.fstride + o] = u[q];
            if (Uhalo) Uhalo[q * b.fstride + o] = u[q];  // the stage's output buffer keeps the same halos
        }
    } else {
#pragma unroll
        for (int q = 0; q < 5; q++) u[q] = U[q * b.fstride + o];
        if (Uhalo && (i < 0 || i >= b.nx || oy || oz)) {  // edges, corners, exchanged planes travel unchanged
#pragma unroll
            for (int q = 0; q < 5; q++) Uhalo[q * b.fstride + o] = u[q];
        }
    }
    prim_from_cons(u, c.gm1, w);
#pragma unroll
    for (int q = 0; q < 5; q++) W[q * b.fstride + o] = w[q];
}

// Face halos only (the regions apply_boundary_conditions + communicate fill):
// U there from its folded source, the same values into Uhalo, W = prim(U)
// there.  The interior of W is the previous x-update's output.  Grid:
// (ceil(3 * max face area / 128), 6 regions: x-, x+, y-, y+, z-, z+).
__global__ void __launch_bounds__(128) k_fill_halo(double* __restrict__ W, double* __restrict__ U,
                                                   Box b, Consts c, double* __restrict__ Uhalo) {
    const int ax = blockIdx.y >> 1, hi = blockIdx.y & 1;
    const long long t = (long long)blockIdx.x * 128 + threadIdx.x;
    // on a slab the y and z ghost rows of exchanged x ghost planes are filled too
    const int ilo = x_exchanged(0, b.nx, c) ? -NG : 0, ihi = b.nx + (x_exchanged(1, b.nx, c) ? NG : 0);
    const int nxe = ihi - ilo;
    int i, j, k, layer;
    if (ax == 0) {
        if (t >= 3LL * b.ny * b.nz) return;
        k = (int)(t % b.nz); j = (int)((t / b.nz) % b.ny); layer = (int)(t / ((long long)b.nz * b.ny));
        i = hi ? b.nx + layer : layer - NG;
    } else if (ax == 1) {
        if (t >= 3LL * nxe * b.nz) return;
        k = (int)(t % b.nz); i = ilo + (int)((t / b.nz) % nxe); layer = (int)(t / ((long long)b.nz * nxe));
        j = hi ? b.ny + layer : layer - NG;
    } else {
        if (t >= 3LL * nxe * b.ny) return;
        layer = (int)(t % 3); j = (int)((t / 3) % b.ny); i = ilo + (int)(t / (3LL * b.ny));
        k = hi ? b.nz + layer : layer - NG;
    }
    const long long o = b.at(i + NG, j + NG, k + NG);
    double u[5], w[5];
    if (ax == 0 && x_exchanged(hi, b.nx, c)) {
        // a neighbour's cells, already in place
#pragma unroll
        for (int q = 0; q < 5; q++) {
            u[q] = U[q * b.fstride + o];
            if (Uhalo) Uhalo[q * b.fstride + o] = u[q];
        }
    } else {
        const int si = ax == 0 ? fold(i, b.nx, c.periodic[0]) : i;
        const int sj = ax == 1 ? fold(j, b.ny, c.periodic[1]) : j;
        const int sk = ax == 2 ? fold(k, b.nz, c.periodic[2]) : k;
        const long long src = b.at(si + NG, sj + NG, sk + NG);
#pragma unroll
        for (int q = 0; q < 5; q++) {
            u[q] = U[q * b.fstride + src];
            U[q * b.fstride + o] = u[q];
            if (Uhalo) Uhalo[q * b.fstride + o] = u[q];
        }
    }
    prim_from_cons(u, c.gm1, w);
#pragma unroll
    for (int q = 0; q < 5; q++) W[q * b.fstride + o] = w[q];
}

// ---------------------------------------------------------------------------
// WENO-5 face fluxes (device functions in ns_face.cuh)

// Minimum resident blocks per SM requested from the register allocator for the
// face kernels (128 threads each), per form.  Chosen by a sweep on B200 at
// 256^3 (1, 3, 4 for FP64; 1, 5, 6 for FP32 characteristic): the caps trade a
// few spilled registers for 12-20 resident warps instead of 8.
#ifndef NS_FACE_MINB_F64CHAR
#define NS_FACE_MINB_F64CHAR 3
#endif
#ifndef NS_FACE_MINB_F64COMP
#define NS_FACE_MINB_F64COMP 4
#endif
#ifndef NS_FACE_MINB_F32CHAR
#define NS_FACE_MINB_F32CHAR 5
#endif
#ifndef NS_FACE_MINB_F32COMP
#define NS_FACE_MINB_F32COMP 1
#endif
template <bool CHAR, typename T>
struct FaceMinBlocks {
    static constexpr int value = sizeof(T) == 8 ? (CHAR ? NS_FACE_MINB_F64CHAR : NS_FACE_MINB_F64COMP)
                                                : (CHAR ? NS_FACE_MINB_F32CHAR : NS_FACE_MINB_F32COMP);
};

// WONLY (time steps, where W = prim(U)): the stencil reads W only and forms U =
// cons(W), half the loads; operator calls read the caller's U as given.
template <int DIR, bool CHAR, bool BORGES, bool PHYS, typename T, typename TF, bool WONLY>
__device__ __forceinline__ void face_at(const double* __restrict__ W, const double* __restrict__ U,
                                        const Box& b, const Consts& c, TF* __restrict__ F,
                                        const FaceBox& fb, int aa, int bb, int kk) {
    long long step;
    long long o0 = face_origin<DIR>(b, aa, bb, kk, step);
    T fL[5][5], fR[5][5], wa[5];
    if constexpr (WONLY) {
        auto ld = [&](int s, T w[5], T u[5]) {
            const long long os = o0 + s * step;
#pragma unroll
            for (int q = 0; q < 5; q++) w[q] = W[q * b.fstride + os];
            cons_from_prim(w, c.inv_gm1, u);
        };
        face_stencil_from<DIR, CHAR, PHYS, T>(ld, c, fL, fR, wa);
    } else {
        face_stencil<DIR, CHAR, PHYS, T>(W, U, b, c, o0, step, fL, fR, wa);
    }
    T out[5];
    if constexpr (!CHAR)
        face_comp<T, BORGES>(fL, fR, out);
    else
        face_char<DIR, PHYS, T, BORGES>(fL, fR, wa, T(c.gamma), T(c.inv_gm1), out);
    long long fo = fb.at(aa, bb, kk);
#pragma unroll
    for (int q = 0; q < 5; q++) F[q * fb.fstride + fo] = TF(out[q]);
}

// Faces of one (i, j) tile row of 32 k-faces per warp, 4 rows per block.  Along
// y and z the last face plane (j = ny, k = nz) is left to k_face_flux_tail: as
// a 33rd k-face or a 4th-of-4 row it would occupy a whole block for one live
// lane or warp per block.
template <int DIR, bool CHAR, bool BORGES, bool PHYS, typename T, typename TF, bool WONLY = false>
__global__ void __launch_bounds__(128, FaceMinBlocks<CHAR, T>::value)
    k_face_flux(const double* __restrict__ W, const double* __restrict__ U, Box b, Consts c,
                TF* __restrict__ F, FaceBox fb, int aa0) {
    int kk = blockIdx.x * 32 + threadIdx.x;
    int bb = blockIdx.y * 4 + threadIdx.y;
    int aa = blockIdx.z + aa0;
    if (kk >= fb.n2 - (DIR == 2) || bb >= fb.n1 - (DIR == 1)) return;
    face_at<DIR, CHAR, BORGES, PHYS, T, TF, WONLY>(W, U, b, c, F, fb, aa, bb, kk);
}

// The last face plane along y (j = ny, threads along k) or z (k = nz, threads
// along j), one face per thread.
template <int DIR, bool CHAR, bool BORGES, bool PHYS, typename T, typename TF, bool WONLY = false>
__global__ void __launch_bounds__(128, FaceMinBlocks<CHAR, T>::value)
    k_face_flux_tail(const double* __restrict__ W, const double* __restrict__ U, Box b, Consts c,
                     TF* __restrict__ F, FaceBox fb, int aa0) {
    static_assert(DIR > 0, "x-faces have no tail plane");
    const int r = blockIdx.x * 128 + threadIdx.x, aa = blockIdx.y + aa0;
    if (r >= (DIR == 1 ? fb.n2 : fb.n1)) return;
    const int bb = DIR == 1 ? fb.n1 - 1 : r, kk = DIR == 1 ? r : fb.n2 - 1;
    face_at<DIR, CHAR, BORGES, PHYS, T, TF, WONLY>(W, U, b, c, F, fb, aa, bb, kk);
}

// ---------------------------------------------------------------------------
// centered viscous terms, reference semantics (CenteredDiffusion::compute_residual,
// src/diffusion_schemes/centered_diffusion.cpp:70-182 with the stress helpers of
// diffusion_scheme.cpp:3-58; dmu = 0 terms dropped, which is exact).
//   - d2/dy2 applies the x-stencil scaled by 1/dy^2 (cd-n.cpp:77)
//   - Tauyy = tauxx (:143); the x work term uses Tauxy*dv_dy (:148);
//     the y heat-flux term multiplies by 1 where the pressure belongs (:166)
//   - 2D terms only; rhoW untouched (:173-176)
//   - mixed derivatives differentiate first derivatives that are zero outside
//     the interior along a non-periodic axis (derivative halos are only filled
//     by the periodic exchange, :22-24)

template <int H, typename TV>
__device__ __forceinline__ void viscous_reference(const double* __restrict__ W, const Box& b,
                                                  const Consts& c, int i, int j, int k, TV r[5]) {
    const long long fs = b.fstride;
    const long long sx = (long long)b.NY * b.NZp, sy = b.NZp;
    const long long o = b.at(i + NG, j + NG, k + NG);
    TV cx1[2 * H + 1], cy1[2 * H + 1], cxx[2 * H + 1], cyy[2 * H + 1];
#pragma unroll
    for (int t = 0; t <= 2 * H; t++) {
        cx1[t] = TV(c.df[3 - H + t] * c.inv_dx);
        cy1[t] = TV(c.df[3 - H + t] * c.inv_dy);
        cxx[t] = TV(c.ddf[3 - H + t] * c.inv_dx * c.inv_dx);
        cyy[t] = TV(c.ddf[3 - H + t] * c.inv_dy * c.inv_dy);
    }
    // first and second derivatives of rho, p, u, v at the cell
    TV Dx[4], Dy[4], Dxx[4], Dyy[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        TV sx1 = 0, sy1 = 0, sxx = 0, syy = 0;
#pragma unroll
        for (int t = 0; t <= 2 * H; t++) {
            TV wx = TV(W[q * fs + o + (t - H) * sx]);
            TV wy = TV(W[q * fs + o + (t - H) * sy]);
            if (t != H) { sx1 += wx * cx1[t]; sy1 += wy * cy1[t]; }
            sxx += wx * cxx[t];
            syy += wx * cyy[t];
        }
        Dx[q] = sx1; Dy[q] = sy1; Dxx[q] = sxx; Dyy[q] = syy;
    }
    // mixed derivatives of u (q=2) and v (q=3)
    TV Dxy[2], Dyx[2];
#pragma unroll
    for (int v = 0; v < 2; v++) {
        const int q = 2 + v;
        TV sxy = 0, syx = 0;
#pragma unroll
        for (int s = 0; s <= 2 * H; s++) {
            if (s == H) continue;
            // The loads run unconditionally from the wrapped (always valid) row or
            // column, so that they issue together; a term outside a non-periodic
            // axis is then dropped by a select.
            // d/dy of (d/dx W) at row j+s-H
            const int jj = j + s - H;
            {
                const int jw = fold(jj, b.ny, 1);
                const long long ob = b.at(i + NG, jw + NG, k + NG);
                TV dx = 0;
#pragma unroll
                for (int t = 0; t <= 2 * H; t++)
                    if (t != H) dx += TV(W[q * fs + ob + (t - H) * sx]) * cx1[t];
                if ((jj >= 0 && jj < b.ny) || c.periodic[1]) sxy += dx * cy1[s];
            }
            // d/dx of (d/dy W) at column i+s-H
            const int ii = i + s - H;
            {
                const int iw = c.ext_x ? ii : fold(ii, b.nx, 1);
                const long long ob = b.at(iw + NG, j + NG, k + NG);
                TV dy = 0;
#pragma unroll
                for (int t = 0; t <= 2 * H; t++)
                    if (t != H) dy += TV(W[q * fs + ob + (t - H) * sy]) * cy1[t];
                if (x_inside(ii, b.nx, c)) syx += dy * cx1[s];
            }
        }
        Dxy[v] = sxy; Dyx[v] = syx;
    }
    viscous_reference_terms<TV>(Dx, Dy, Dxx, Dyy, Dxy, Dyx, TV(W[2 * fs + o]), TV(W[3 * fs + o]),
                                TV(W[1 * fs + o]), TV(W[o]), c, r);
}

// Reference semantics: the terms of viscous_reference above, in the same
// arithmetic order, from an accessor at(q, ox, oy) of W at offsets ox along x
// and oy along y of the cell (the TMA-marched kernel reads its shared-memory
// planes through it).  The mixed derivatives read the rows/columns the
// per-thread kernel wraps to; the box holds them as the filled face halos.
template <int H, typename TV, typename At>
__device__ __forceinline__ void viscous_reference_core(At at, const Box& b, const Consts& c, int i, int j,
                                                       TV r[5]) {
    TV cx1[2 * H + 1], cy1[2 * H + 1], cxx[2 * H + 1], cyy[2 * H + 1];
#pragma unroll
    for (int t = 0; t <= 2 * H; t++) {
        cx1[t] = TV(c.df[3 - H + t] * c.inv_dx);
        cy1[t] = TV(c.df[3 - H + t] * c.inv_dy);
        cxx[t] = TV(c.ddf[3 - H + t] * c.inv_dx * c.inv_dx);
        cyy[t] = TV(c.ddf[3 - H + t] * c.inv_dy * c.inv_dy);
    }
    TV Dx[4], Dy[4], Dxx[4], Dyy[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        TV sx1 = 0, sy1 = 0, sxx = 0, syy = 0;
#pragma unroll
        for (int t = 0; t <= 2 * H; t++) {
            TV wx = TV(at(q, t - H, 0));
            TV wy = TV(at(q, 0, t - H));
            if (t != H) { sx1 += wx * cx1[t]; sy1 += wy * cy1[t]; }
            sxx += wx * cxx[t];
            syy += wx * cyy[t];
        }
        Dx[q] = sx1; Dy[q] = sy1; Dxx[q] = sxx; Dyy[q] = syy;
    }
    TV Dxy[2], Dyx[2];
#pragma unroll
    for (int v = 0; v < 2; v++) {
        const int q = 2 + v;
        TV sxy = 0, syx = 0;
#pragma unroll
        for (int s = 0; s <= 2 * H; s++) {
            if (s == H) continue;
            const int jj = j + s - H;
            {
                TV dx = 0;
#pragma unroll
                for (int t = 0; t <= 2 * H; t++)
                    if (t != H) dx += TV(at(q, t - H, s - H)) * cx1[t];
                if ((jj >= 0 && jj < b.ny) || c.periodic[1]) sxy += dx * cy1[s];
            }
            const int ii = i + s - H;
            {
                TV dy = 0;
#pragma unroll
                for (int t = 0; t <= 2 * H; t++)
                    if (t != H) dy += TV(at(q, s - H, t - H)) * cy1[t];
                if (x_inside(ii, b.nx, c)) syx += dy * cx1[s];
            }
        }
        Dxy[v] = sxy; Dyx[v] = syx;
    }
    viscous_reference_terms<TV>(Dx, Dy, Dxx, Dyy, Dxy, Dyx, TV(at(2, 0, 0)), TV(at(3, 0, 0)), TV(at(1, 0, 0)),
                                TV(at(0, 0, 0)), c, r);
}

// Physical semantics: the full 3D viscous terms of viscous_physical below, in
// the same arithmetic order (p / rho by div_pos_nr, within an ulp of the
// division), from two accessors of W around the cell (the
// TMA-marched kernel reads its shared-memory planes through them; the
// per-thread kernel keeps its own loads, which compile to fewer registers):
// ld1(q, ax, t) = field q at offset t - H along axis ax, ld2(q, a, s, bx, t) =
// field q at offsets s - H along a and t - H along bx (mixed derivatives).
// All axis loops unroll at compile time (2D skips the z terms at run time).
template <int H, typename TV, typename Ld1, typename Ld2>
__device__ __forceinline__ void viscous_physical_core(Ld1 ld1, Ld2 ld2, const Consts& c, TV r[5]) {
    constexpr int NS = 2 * H + 1;
    const bool three = c.dim == 3;
    const double inv[3] = {c.inv_dx, c.inv_dy, c.inv_dz};
    TV c1[3][NS], c2[3][NS];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int t = 0; t < NS; t++) {
            c1[a][t] = TV(c.df[3 - H + t] * inv[a]);
            c2[a][t] = TV(c.ddf[3 - H + t] * inv[a] * inv[a]);
        }
    TV gu[3][3], lap[3], gdiv[3], lapT = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        lap[a] = 0;
        gdiv[a] = 0;
#pragma unroll
        for (int bx = 0; bx < 3; bx++) gu[a][bx] = 0;
    }
#pragma unroll
    for (int bx = 0; bx < 3; bx++) {
        if (bx == 2 && !three) continue;
#pragma unroll
        for (int t = 0; t < NS; t++) {
            // p / rho (rho > 0): the Newton-Raphson quotient of the WENO weights in FP64
            TV T;
            if constexpr (sizeof(TV) == 8) T = div_pos_nr(ld1(1, bx, t), ld1(0, bx, t));
            else T = TV(ld1(1, bx, t)) / TV(ld1(0, bx, t));
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const TV va = TV(ld1(2 + a, bx, t));
                if (t != H) gu[a][bx] += va * c1[bx][t];
                lap[a] += va * c2[bx][t];
                if (a == bx) gdiv[a] += va * c2[bx][t];
            }
            lapT += T * c2[bx][t];
        }
    }
    // grad(div u)_a += d/dx_a (d u_b / dx_b) for b != a
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int bx = 0; bx < 3; bx++) {
            if (a == bx || ((a == 2 || bx == 2) && !three)) continue;
            TV acc = 0;
#pragma unroll
            for (int s = 0; s < NS; s++) {
                if (s == H) continue;
                TV inner = 0;
#pragma unroll
                for (int t = 0; t < NS; t++) {
                    if (t == H) continue;
                    inner += TV(ld2(2 + bx, a, s, bx, t)) * c1[bx][t];
                }
                acc += inner * c1[a][s];
            }
            gdiv[a] += acc;
        }
    const TV mu = TV(c.mu), lamb = TV(c.lamb);
    const TV uv[3] = {TV(ld1(2, 0, H)), TV(ld1(3, 0, H)), TV(ld1(4, 0, H))};
    const TV div = gu[0][0] + gu[1][1] + gu[2][2];
    TV work = 0, diss = 0, mom[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        mom[a] = mu * lap[a] + (mu + lamb) * gdiv[a];
        work += uv[a] * mom[a];
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int bx = 0; bx < 3; bx++) {
            const TV tab = mu * (gu[a][bx] + gu[bx][a]) + (a == bx ? lamb * div : TV(0));
            diss += tab * gu[a][bx];
        }
    r[2] -= mom[0];
    r[3] -= mom[1];
    r[4] -= mom[2];
    r[1] -= work + diss + TV(c.heat) * mu * lapT;
}

// Physical semantics: full 3D viscous stress and heat flux with constant mu
// (no reference counterpart).  Derivatives along one axis read the
// boundary-filled W as it is (ghost cells included); a mixed derivative also
// reads edge and corner cells, which no fill writes, so its offsets are folded
// back into the interior along each axis (periodic wrap or Neumann clamp; a
// slab's x ghost planes are the neighbours' cells and stay).  All axis loops
// unroll at compile time (2D skips the z terms at run time) and the folded
// offsets are formed once per axis.
template <int H, typename TV>
__device__ __forceinline__ void viscous_physical(const double* __restrict__ W, const Box& b,
                                                 const Consts& c, int i, int j, int k, TV r[5]) {
    constexpr int NS = 2 * H + 1;
    const long long fs = b.fstride;
    const long long st3[3] = {(long long)b.NY * b.NZp, (long long)b.NZp, 1};
    const long long o = b.at(i + NG, j + NG, k + NG);
    const bool three = c.dim == 3;
    const double inv[3] = {c.inv_dx, c.inv_dy, c.inv_dz};
    const int n3[3] = {b.nx, b.ny, b.nz};
    const int c3[3] = {i, j, k};
    // offsets of the folded stencil cells along each axis, and the CD coefficients
    long long off[3][NS];
    TV c1[3][NS], c2[3][NS];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int t = 0; t < NS; t++) {
            const int v = c3[a] + t - H;
            const int f = (a == 0) ? fold_x(v, n3[0], c) : fold(v, n3[a], c.periodic[a]);
            off[a][t] = (long long)(f - c3[a]) * st3[a];
            c1[a][t] = TV(c.df[3 - H + t] * inv[a]);
            c2[a][t] = TV(c.ddf[3 - H + t] * inv[a] * inv[a]);
        }
    TV gu[3][3], lap[3], gdiv[3], lapT = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        lap[a] = 0;
        gdiv[a] = 0;
#pragma unroll
        for (int bx = 0; bx < 3; bx++) gu[a][bx] = 0;
    }
#pragma unroll
    for (int bx = 0; bx < 3; bx++) {
        if (bx == 2 && !three) continue;
#pragma unroll
        for (int t = 0; t < NS; t++) {
            const long long oo = o + (t - H) * st3[bx];
            const TV T = TV(W[1 * fs + oo]) / TV(W[oo]);
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const TV va = TV(W[(2 + a) * fs + oo]);
                if (t != H) gu[a][bx] += va * c1[bx][t];
                lap[a] += va * c2[bx][t];
                if (a == bx) gdiv[a] += va * c2[bx][t];
            }
            lapT += T * c2[bx][t];
        }
    }
    // grad(div u)_a += d/dx_a (d u_b / dx_b) for b != a
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int bx = 0; bx < 3; bx++) {
            if (a == bx || ((a == 2 || bx == 2) && !three)) continue;
            TV acc = 0;
#pragma unroll
            for (int s = 0; s < NS; s++) {
                if (s == H) continue;
                TV inner = 0;
#pragma unroll
                for (int t = 0; t < NS; t++) {
                    if (t == H) continue;
                    inner += TV(W[(2 + bx) * fs + o + off[a][s] + off[bx][t]]) * c1[bx][t];
                }
                acc += inner * c1[a][s];
            }
            gdiv[a] += acc;
        }
    const TV mu = TV(c.mu), lamb = TV(c.lamb);
    const TV uv[3] = {TV(W[2 * fs + o]), TV(W[3 * fs + o]), TV(W[4 * fs + o])};
    const TV div = gu[0][0] + gu[1][1] + gu[2][2];
    TV work = 0, diss = 0, mom[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        mom[a] = mu * lap[a] + (mu + lamb) * gdiv[a];
        work += uv[a] * mom[a];
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int bx = 0; bx < 3; bx++) {
            const TV tab = mu * (gu[a][bx] + gu[bx][a]) + (a == bx ? lamb * div : TV(0));
            diss += tab * gu[a][bx];
        }
    r[2] -= mom[0];
    r[3] -= mom[1];
    r[4] -= mom[2];
    r[1] -= work + diss + TV(c.heat) * mu * lapT;
}

// ---------------------------------------------------------------------------
// cell update: R = sum_d (f_d(+) - f_d(-))/d  (+ viscous), then
//   MODE_STAGE: U = U0*m1 + U*m2 + R*(mc*dt)    (TimeScheme::substep, time_scheme.cpp:72-96)
//   MODE_RHS  : Rout += R
// dt = CFL * min(1e10, reduced minimum) (time_scheme.cpp:98-136).

// The update kernel is memory-latency bound; 8 resident blocks (64 registers)
// matched the compiler's own choice and beat looser bounds in a B200 sweep.
#ifndef NS_UPDATE_MINB
#define NS_UPDATE_MINB 8
#endif
template <int MODE, int H, bool PHYS, typename TF, typename TV>
__global__ void __launch_bounds__(128, NS_UPDATE_MINB) k_update(const double* __restrict__ W, double* __restrict__ U,
                                                const double* __restrict__ U0,
                                                const TF* __restrict__ Fx, const TF* __restrict__ Fy,
                                                const TF* __restrict__ Fz, Box b, FaceBox fx,
                                                FaceBox fy, FaceBox fz, Consts c, int flags,
                                                const unsigned long long* __restrict__ slot,
                                                double m1, double m2, double mc,
                                                double* __restrict__ Rout, double* __restrict__ clock) {
    int k = blockIdx.x * 32 + threadIdx.x;
    int j = blockIdx.y * 4 + threadIdx.y;
    int i = blockIdx.z;
    if (k >= b.nz || j >= b.ny) return;
    double r[5] = {0, 0, 0, 0, 0};
    if (flags & UPD_CONV) {
#pragma unroll
        for (int q = 0; q < 5; q++) {
            r[q] += (double(Fx[q * fx.fstride + fx.at(i + 1, j, k)]) -
                     double(Fx[q * fx.fstride + fx.at(i, j, k)])) * c.inv_dx;
            r[q] += (double(Fy[q * fy.fstride + fy.at(i, j + 1, k)]) -
                     double(Fy[q * fy.fstride + fy.at(i, j, k)])) * c.inv_dy;
            if (flags & UPD_CONVZ)
                r[q] += (double(Fz[q * fz.fstride + fz.at(i, j, k + 1)]) -
                         double(Fz[q * fz.fstride + fz.at(i, j, k)])) * c.inv_dz;
        }
    }
    if constexpr (H > 0) {
        TV rv[5] = {0, 0, 0, 0, 0};
        if constexpr (PHYS)
            viscous_physical<H, TV>(W, b, c, i, j, k, rv);
        else
            viscous_reference<H, TV>(W, b, c, i, j, k, rv);
#pragma unroll
        for (int q = 1; q < 5; q++) r[q] += double(rv[q]);
    }
    long long o = b.at(i + NG, j + NG, k + NG);
    if constexpr (MODE == MODE_STAGE) {
        double mn = __longlong_as_double((long long)*slot);
        double dt = fmin(1e10, mn) * c.cfl;
        double m3 = mc * dt;
        if (clock && (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0) {
            clock[0] = dt;
            clock[1] += dt;
        }
#pragma unroll
        for (int q = 0; q < 5; q++) {
            long long a = q * b.fstride + o;
            U[a] = (U0[a] * m1) + (U[a] * m2) + (r[q] * m3);
        }
    } else {
        if (flags & UPD_OVERWRITE) {
#pragma unroll
            for (int q = 0; q < 5; q++) Rout[q * b.fstride + o] = r[q];
        } else {
#pragma unroll
            for (int q = 0; q < 5; q++) Rout[q * b.fstride + o] += r[q];
        }
    }
}

// ---------------------------------------------------------------------------
// Viscous terms of every interior cell (residual components 1..4, component 0
// is zero) into V: plane q-1 of stride vs, cell ((i ny + j) nz + k).  A
// stencil kernel of its own at full occupancy: inside the x-march its loads sat
// on the latency path of a 12-warp-per-SM kernel (0.75 ms of 2.47 ms per stage
// at 256^3, CD-2).
template <int H, bool PHYS>
__global__ void __launch_bounds__(128) k_viscous(const double* __restrict__ W, Box b, Consts c,
                                                 double* __restrict__ V, long long vs) {
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 4 + threadIdx.y, i = blockIdx.z;
    if (k >= b.nz || j >= b.ny) return;
    double rv[5] = {0, 0, 0, 0, 0};
    if constexpr (PHYS)
        viscous_physical<H, double>(W, b, c, i, j, k, rv);
    else
        viscous_reference<H, double>(W, b, c, i, j, k, rv);
    const long long e = ((long long)i * b.ny + j) * b.nz + k;
#pragma unroll
    for (int q = 1; q < 5; q++) V[(q - 1) * vs + e] = rv[q];
}

// Physical semantics: the same terms from planes of W that the TMA unit loads
// into a ring while the block marches VISC_LX cells along x.  A block owns 4
// rows x 32 columns; one plane is the box of ViscTile<H> (5 fields; 8.2, 12.2
// and 15.2 KB for CD-2, 4, 6), so each cell of W crosses L2 once per block
// instead of once per stencil.  The ring holds the 2H+1 planes of the current
// cell and, for CD-2 and CD-4, the next plane in flight; CD-6 keeps 7 slots
// (two blocks per SM) and loads the next plane as the last one is released.
// A cell within H cells of the boundary along two axes or more needs folded
// edge or corner ghost cells for its mixed derivatives, which no fill writes
// and so the box does not hold: it reads the device state like k_viscous.  Waits are
// bounded (the error word receives 1 and the block ends).
#ifndef NS_VISC_LX
#define NS_VISC_LX 32
#endif
constexpr int VISC_LX = NS_VISC_LX;

template <int H>
struct ViscRing {
    using VT = ViscTile<H>;
    static constexpr int QS = VT::BZ * VT::BY, ELEMS = 5 * QS;
    static constexpr int STRIDE = (ELEMS + 15) / 16 * 16;  // 128-byte aligned slots
    static constexpr uint32_t BYTES = ELEMS * 8;
    static constexpr int LEAD = H < 3 ? 1 : 0;             // planes in flight beyond the stencil
    static constexpr int NSLOT = 2 * H + 1 + LEAD;
    // the ring, then its mbarriers: no static shared memory, so the dynamic ring
    // starts at the window's base (TMA writes want 128-byte aligned destinations)
    static constexpr size_t smem = (size_t)NSLOT * STRIDE * 8 + NSLOT * 8;
    static constexpr int MINB = H == 1 ? 4 : (H == 2 ? 3 : 2);
};

template <int H, bool PHYS>
__global__ void __launch_bounds__(128, ViscRing<H>::MINB)
    k_viscous_tma(const __grid_constant__ CUtensorMap map, const double* __restrict__ W, Box b, Consts c,
                  double* __restrict__ V, long long vs, unsigned long long* __restrict__ err, int seg0) {
    using VT = ViscTile<H>;
    using VR = ViscRing<H>;
    constexpr int NSLOT = VR::NSLOT, STRIDE = VR::STRIDE, QS = VR::QS, BZ = VT::BZ;
    extern __shared__ __align__(128) double vring[];  // [NSLOT][5][BY][BZ], then NSLOT mbarriers
    unsigned long long* full = reinterpret_cast<unsigned long long*>(vring + NSLOT * STRIDE);
    const int lane = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + lane;
    if (tc::smem_u32(vring) & 127u) {  // a TMA destination must be 128-byte aligned: report, touch nothing
        if (tid == 0) atomicOr(err, 2ull);
        return;
    }
    const int k0 = blockIdx.x * 32, j0 = blockIdx.y * 4, x0 = (blockIdx.z + seg0) * VISC_LX;
    const int x1 = min(x0 + VISC_LX, b.nx);
    const int k = k0 + lane, j = j0 + ty;
    const bool live = k < b.nz && j < b.ny;
    // plane p (x0 - H <= p <= x1 - 1 + H) is the (p - x0 + H)-th load of the block
    auto slot = [&](int p) { return (p - x0 + H) % NSLOT; };
    auto bar = [&](int p) { return tc::smem_u32(&full[slot(p)]); };
    auto par = [&](int p) { return (uint32_t)(((p - x0 + H) / NSLOT) & 1); };
    auto issue = [&](int p) {
        mbar_expect_tx(bar(p), VR::BYTES);
        tma_load_4d(tc::smem_u32(vring + slot(p) * STRIDE), &map, k0 + VT::Z0, j0 + NG - H, p + NG, 0, bar(p));
    };
    if (tid == 0)
        for (int q = 0; q < NSLOT; q++) tc::mbar_init(tc::smem_u32(&full[q]), 1);
    __syncthreads();
    const int last = x1 - 1 + H;  // the last plane the block reads
    if (tid == 0)
        for (int p = x0 - H; p <= min(x0 + H + VR::LEAD, last); p++) issue(p);
    bool ok = true;
    for (int p = x0 - H; p < x0 + H; p++) ok = ok && tc::mbar_wait(bar(p), par(p), kTilePolls);
    int waited = ok ? x0 + H - 1 : x0 - H - 1;  // planes up to this one have landed
    // within H cells of the boundary along two axes or more, a mixed derivative
    // reaches an edge or corner ghost cell
    const int nbjk = (j < H || j >= b.ny - H) + (k < H || k >= b.nz - H);
    const int cc = (ty + H) * BZ + lane + VT::C0;
    for (int i = x0; i < x1; i++) {
        if (ok && i + H > waited) {
            ok = tc::mbar_wait(bar(i + H), par(i + H), kTilePolls);
            if (ok) waited = i + H;
        }
        if (ok && live) {
            double rv[5] = {0, 0, 0, 0, 0};
            if (nbjk + (i < H || i >= b.nx - H) >= 2) {
                if constexpr (PHYS)
                    viscous_physical<H, double>(W, b, c, i, j, k, rv);
                else
                    viscous_reference<H, double>(W, b, c, i, j, k, rv);
            } else if constexpr (!PHYS) {
                const double* P[2 * H + 1];
#pragma unroll
                for (int s = 0; s <= 2 * H; s++) P[s] = vring + slot(i - H + s) * STRIDE;
                auto at = [&](int q, int ox, int oy) { return P[H + ox][q * QS + cc + oy * BZ]; };
                viscous_reference_core<H, double>(at, b, c, i, j, rv);
            } else {
                const double* P[2 * H + 1];
#pragma unroll
                for (int s = 0; s <= 2 * H; s++) P[s] = vring + slot(i - H + s) * STRIDE;
                auto at = [&](int q, int ox, int oy, int oz) { return P[H + ox][q * QS + cc + oy * BZ + oz]; };
                auto ld1 = [&](int q, int ax, int t) {
                    const int d = t - H;
                    return at(q, ax == 0 ? d : 0, ax == 1 ? d : 0, ax == 2 ? d : 0);
                };
                auto ld2 = [&](int q, int a, int s, int bx, int t) {
                    int o[3] = {0, 0, 0};
                    o[a] += s - H;
                    o[bx] += t - H;
                    return at(q, o[0], o[1], o[2]);
                };
                viscous_physical_core<H, double>(ld1, ld2, c, rv);
            }
            const long long e = ((long long)i * b.ny + j) * b.nz + k;
#pragma unroll
            for (int q = 1; q < 5; q++) V[(q - 1) * vs + e] = rv[q];
        }
        // every thread is done with plane i - H (and agrees on whether a wait ran out)
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicOr(err, 1ull);
                // the loads still in flight: planes waited + 1 .. the last one issued
                const int issued = min(i + H + VR::LEAD, last);
                for (int p = waited + 1; p <= issued; p++) tc::mbar_wait(bar(p), par(p), kTilePolls);
            }
            __syncthreads();
            return;
        }
        const int next = i + H + 1 + VR::LEAD;  // into the slot of plane i - H
        if (tid == 0 && next <= last) issue(next);
    }
}

// ---------------------------------------------------------------------------
// FP64 stage, last kernel: x-face fluxes marched along x with the cell update of
// each cell as soon as both of its x-faces are known (same face and update
// arithmetic as k_face_flux<0> + k_update).  The x-face array never reaches
// HBM, and the update's loads (U0, U, the y- and z-face fluxes, W for the
// viscous terms) overlap the x-faces' FP64 work.  U_out is a second buffer:
// other threads still read U's x-neighbours for their stencils.  (A variant that
// kept each thread's 6-cell W stencil in a shared ring, loading every cell once,
// ran 5-24% slower on B200 at 256^3, with 70 KB of shared memory per block and
// three blocks per SM leaving about 30 KB of L1 for everything else.)

// Cells a thread marches: 24 ran 3% faster than 32 at 256^3 (more, shorter
// blocks balance the SMs better; the extra x-face per block costs less), 20
// the same as 24, 43 and 52 slower.
#ifndef NS_XMARCH_L
#define NS_XMARCH_L 24
#endif
//
// LAST (third stage): the next step's start as well -- W = prim(U_out) for its
// CFL minimum (time_scheme.cpp:69, 98-136) into slot_next and U0 = cons(W)
// (the W -> U round trip of time_scheme.cpp:124); U_out itself stays the raw
// stage result, as the reference's U holds it between steps.  In the first stage U
// and U0 are one buffer, only read; U0 is written in the third stage only, where
// it is not U (so the restrict qualifiers hold).
// Resident blocks per SM requested for the characteristic-wise march: the
// reference semantics' march ran 7% faster at 2 (255 registers, no spills) than
// at 3 (168 registers, spills), the physical semantics' 13% slower (B200, 256^3).
template <bool CHAR, bool PHYS>
struct XupdMinBlocks {
    static constexpr int value = CHAR ? (PHYS ? 3 : 2) : FaceMinBlocks<false, double>::value;
};
template <bool CHAR, bool BORGES, bool PHYS, int H, bool LAST>
__global__ void __launch_bounds__(128, XupdMinBlocks<CHAR, PHYS>::value)
    k_xface_update(const double* __restrict__ W, const double* __restrict__ U, double* __restrict__ U0,
                   double* __restrict__ Uout, double* __restrict__ Wn,
                   const double* __restrict__ Fy, const double* __restrict__ Fz,
                   const double* __restrict__ V, long long vs, Box b, FaceBox fy,
                   FaceBox fz, Consts c, int flags, const unsigned long long* __restrict__ slot,
                   unsigned long long* __restrict__ slot_next, double m1, double m2, double mc,
                   double* __restrict__ clock) {
    __shared__ double fprev[5][128];  // the x-face below the thread's next cell
    // the update's operands of cell i (U0, U, the two y- and two z-faces, the
    // viscous terms from k_viscous), copied in while the thread computes x-face
    // i+1; each thread reads only its own
    __shared__ double opnd[H > 0 ? 34 : 30][128];
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 4 + threadIdx.y;
    const int t = threadIdx.y * 32 + threadIdx.x;
    const int x0 = blockIdx.z * NS_XMARCH_L;
    // threads outside the grid march no cells but join the block reduction of LAST
    const int x1 = (k < b.nz && j < b.ny) ? min(x0 + NS_XMARCH_L, b.nx) : x0 - 1;
    double best = INFINITY;
    const double dt = fmin(1e10, __longlong_as_double((long long)*slot)) * c.cfl;
    const double m3 = mc * dt;
    if (clock && (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0) {
        clock[0] = dt;
        clock[1] += dt;
    }
    // x-face a (between cells a-1 and a) of this thread's column.  The stencil
    // reads W only and forms U = cons(W) (rounding-level difference from the
    // stage's U): half the cached working set of a march, which keeps the
    // re-read stencil cells in L1.
    auto xface = [&](int a, double out[5]) {
        long long step;
        const long long o0 = face_origin<0>(b, a, j, k, step);
        auto ld = [&](int s, double w[5], double u[5]) {
            const long long os = o0 + s * step;
#pragma unroll
            for (int q = 0; q < 5; q++) w[q] = W[q * b.fstride + os];
            cons_from_prim(w, c.inv_gm1, u);
        };
        double fL[5][5], fR[5][5], wa[5];
        face_stencil_from<0, CHAR, PHYS, double>(ld, c, fL, fR, wa);
        if constexpr (!CHAR)
            face_comp<double, BORGES>(fL, fR, out);
        else
            face_char<0, PHYS, double, BORGES>(fL, fR, wa, c.gamma, c.inv_gm1, out);
    };
    const bool convz = flags & UPD_CONVZ;
    // one face call site: the pass i = x0 - 1 only forms the first x-face
    for (int i = x0 - 1; i < x1; i++) {
        const long long o = b.at(i + NG, j + NG, k + NG);
        if (i >= x0) {
#pragma unroll
            for (int q = 0; q < 5; q++) {
                cp_async8(&opnd[q][t], U0 + q * b.fstride + o);
                cp_async8(&opnd[5 + q][t], U + q * b.fstride + o);
                cp_async8(&opnd[10 + q][t], Fy + q * fy.fstride + fy.at(i, j, k));
                cp_async8(&opnd[15 + q][t], Fy + q * fy.fstride + fy.at(i, j + 1, k));
                if (convz) {
                    cp_async8(&opnd[20 + q][t], Fz + q * fz.fstride + fz.at(i, j, k));
                    cp_async8(&opnd[25 + q][t], Fz + q * fz.fstride + fz.at(i, j, k + 1));
                }
            }
            if constexpr (H > 0) {
                const long long e = ((long long)i * b.ny + j) * b.nz + k;
#pragma unroll
                for (int q = 0; q < 4; q++) cp_async8(&opnd[30 + q][t], V + q * vs + e);
            }
            cp_async_commit();
        }
        double f[5];
        xface(i + 1, f);
        if (i < x0) {
#pragma unroll
            for (int q = 0; q < 5; q++) fprev[q][t] = f[q];
            continue;
        }
        cp_async_wait_all();
        // residual in k_update's order: x, y, z differences, then the viscous terms
        double r[5] = {0, 0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < 5; q++) {
            r[q] += (f[q] - fprev[q][t]) * c.inv_dx;
            fprev[q][t] = f[q];
            r[q] += (opnd[15 + q][t] - opnd[10 + q][t]) * c.inv_dy;
            if (convz) r[q] += (opnd[25 + q][t] - opnd[20 + q][t]) * c.inv_dz;
        }
        if constexpr (H > 0) {
#pragma unroll
            for (int q = 1; q < 5; q++) r[q] += opnd[29 + q][t];
        }
        double un[5], w[5];
#pragma unroll
        for (int q = 0; q < 5; q++) {
            un[q] = (opnd[q][t] * m1) + (opnd[5 + q][t] * m2) + (r[q] * m3);
            Uout[q * b.fstride + o] = un[q];
        }
        prim_from_cons(un, c.gm1, w);  // the next stage's W (conservative_to_primitive, time_scheme.cpp)
        if constexpr (LAST) {
            double u0[5];
            const double d = PHYS ? local_dt_physical(w, c) : local_dt(w, c);
            if (d < best) best = d;  // NaN never lowers the minimum (time_scheme.cpp:117)
            cons_from_prim(w, c.inv_gm1, u0);
#pragma unroll
            for (int q = 0; q < 5; q++) U0[q * b.fstride + o] = u0[q];
            prim_from_cons(u0, c.gm1, w);  // the next step's first stage reads prim(U0)
        }
#pragma unroll
        for (int q = 0; q < 5; q++) Wn[q * b.fstride + o] = w[q];
    }
    if constexpr (LAST) block_min_to(best, slot_next);
}

// ---------------------------------------------------------------------------
// error bounds of div_pos_nr against the IEEE quotient and of rsqrt_pos_nr
// against CUDA's rsqrt: n pairs with x log-uniform in [1e-3, 1e3] and d
// log-uniform in [1e-60, 1e60] (SplitMix64 draws); max_ulp[0], max_ulp[1]
// receive the largest distances in units in the last place

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void k_div_check(long long n, unsigned long long seed, unsigned long long* __restrict__ max_ulp) {
    unsigned long long worst = 0, worst_r = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const double u = (splitmix64(seed + 2 * e) >> 11) * 0x1.0p-53;
        const double v = (splitmix64(seed + 2 * e + 1) >> 11) * 0x1.0p-53;
        const double x = exp10(-3.0 + 6.0 * u), d = exp10(-60.0 + 120.0 * v);
        const long long a = __double_as_longlong(div_pos_nr(x, d)), b = __double_as_longlong(x / d);
        const unsigned long long dist = (unsigned long long)(a > b ? a - b : b - a);
        if (dist > worst) worst = dist;
        // 1/sqrt(d) against CUDA's rsqrt (itself within an ulp)
        const long long ra = __double_as_longlong(rsqrt_pos_nr(d)), rb = __double_as_longlong(rsqrt(d));
        const unsigned long long rdist = (unsigned long long)(ra > rb ? ra - rb : rb - ra);
        if (rdist > worst_r) worst_r = rdist;
    }
    atomicMax(max_ulp, worst);
    atomicMax(max_ulp + 1, worst_r);
}

cudaError_t launch_div_check(long long n, unsigned long long seed, unsigned long long* max_ulp, cudaStream_t s) {
    k_div_check<<<256, 256, 0, s>>>(n, seed, max_ulp);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// host <-> device layout transposes (reference AoS [i][j][k][q], unpadded
// (nx+6)(ny+6)(nz+6) x 5  <->  device SoA planes)

__global__ void __launch_bounds__(128) k_aos_to_soa(const double* __restrict__ A, double* __restrict__ S,
                                                    Box b, int ih0) {
    int kh = blockIdx.x * 32 + threadIdx.x;
    int jh = blockIdx.y * 4 + threadIdx.y;
    int ih = blockIdx.z + ih0;
    int NZ = b.nz + 2 * NG;
    if (kh >= NZ || jh >= b.NY) return;
    long long a = (((long long)ih * b.NY + jh) * NZ + kh) * 5;
    long long o = b.at(ih, jh, kh);
#pragma unroll
    for (int q = 0; q < 5; q++) S[q * b.fstride + o] = A[a + q];
}

__global__ void __launch_bounds__(128) k_soa_to_aos(const double* __restrict__ S, double* __restrict__ A,
                                                    Box b, int ih0) {
    int kh = blockIdx.x * 32 + threadIdx.x;
    int jh = blockIdx.y * 4 + threadIdx.y;
    int ih = blockIdx.z + ih0;
    int NZ = b.nz + 2 * NG;
    if (kh >= NZ || jh >= b.NY) return;
    long long a = (((long long)ih * b.NY + jh) * NZ + kh) * 5;
    long long o = b.at(ih, jh, kh);
#pragma unroll
    for (int q = 0; q < 5; q++) A[a + q] = S[q * b.fstride + o];
}

// ---------------------------------------------------------------------------
// slab halo exchange (Communicator::communicate_x_direction, src/communicator.cpp:16-57,
// with the slices of src/containers/array_4d.cpp:39-84): the outer three interior
// planes of one side packed as [q][layer][j][k], interior j and k; unpack writes
// the same layout into the ghost planes of that side.
__global__ void __launch_bounds__(128) k_slab_pack(const double* __restrict__ U, Box b, int side,
                                                   double* __restrict__ buf) {
    const long long n = 3LL * b.ny * b.nz, t = (long long)blockIdx.x * 128 + threadIdx.x;
    if (t >= 5 * n) return;
    const int q = (int)(t / n);
    const long long r = t % n;
    const int layer = (int)(r / ((long long)b.ny * b.nz)), j = (int)((r / b.nz) % b.ny), k = (int)(r % b.nz);
    const int i = side ? b.nx - NG + layer : layer;
    buf[t] = U[q * b.fstride + b.at(i + NG, j + NG, k + NG)];
}

__global__ void __launch_bounds__(128) k_slab_unpack(double* __restrict__ U, Box b, int side,
                                                     const double* __restrict__ buf) {
    const long long n = 3LL * b.ny * b.nz, t = (long long)blockIdx.x * 128 + threadIdx.x;
    if (t >= 5 * n) return;
    const int q = (int)(t / n);
    const long long r = t % n;
    const int layer = (int)(r / ((long long)b.ny * b.nz)), j = (int)((r / b.nz) % b.ny), k = (int)(r % b.nz);
    const int i = side ? b.nx + layer : layer - NG;
    U[q * b.fstride + b.at(i + NG, j + NG, k + NG)] = buf[t];
}

// ---------------------------------------------------------------------------
// global diagnostics over the interior (FP64): sums of conserved variables,
// kinetic energy, enstrophy (second-order central curl), non-finite count.
__global__ void __launch_bounds__(128) k_diagnostics(const double* __restrict__ U, Box b, Consts c,
                                                     double* __restrict__ acc) {
    int k = blockIdx.x * 32 + threadIdx.x;
    int j = blockIdx.y * 4 + threadIdx.y;
    int i = blockIdx.z;
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (k < b.nz && j < b.ny) {
        long long o = b.at(i + NG, j + NG, k + NG);
        double u[5];
        bool bad = false;
#pragma unroll
        for (int q = 0; q < 5; q++) {
            u[q] = U[q * b.fstride + o];
            bad |= !isfinite(u[q]);
        }
        double dV = c.dx * c.dy * c.dz;
        v[0] = u[0] * dV;
        v[1] = u[2] * dV;
        v[2] = u[3] * dV;
        v[3] = u[4] * dV;
        v[4] = u[1] * dV;
        v[5] = 0.5 * (u[2] * u[2] + u[3] * u[3] + u[4] * u[4]) / u[0] * dV;
        // velocity of neighbours through the periodic/clamped index map
        auto vel = [&](int ii, int jj, int kk, int a) {
            ii = fold_x(ii, b.nx, c);
            jj = fold(jj, b.ny, c.periodic[1]);
            kk = fold(kk, b.nz, c.periodic[2]);
            long long oo = b.at(ii + NG, jj + NG, kk + NG);
            return U[(2 + a) * b.fstride + oo] / U[oo];
        };
        double dwdy = (vel(i, j + 1, k, 2) - vel(i, j - 1, k, 2)) * 0.5 * c.inv_dy;
        double dvdz = (vel(i, j, k + 1, 1) - vel(i, j, k - 1, 1)) * 0.5 * c.inv_dz;
        double dudz = (vel(i, j, k + 1, 0) - vel(i, j, k - 1, 0)) * 0.5 * c.inv_dz;
        double dwdx = (vel(i + 1, j, k, 2) - vel(i - 1, j, k, 2)) * 0.5 * c.inv_dx;
        double dvdx = (vel(i + 1, j, k, 1) - vel(i - 1, j, k, 1)) * 0.5 * c.inv_dx;
        double dudy = (vel(i, j + 1, k, 0) - vel(i, j - 1, k, 0)) * 0.5 * c.inv_dy;
        double wx = dwdy - dvdz, wy = dudz - dwdx, wz = dvdx - dudy;
        v[6] = 0.5 * u[0] * (wx * wx + wy * wy + wz * wz) * dV;
        v[7] = bad ? 1.0 : 0.0;
    }
    __shared__ double red[8][4];
    int warp = threadIdx.y;  // blockDim = (32,4): one warp per row
#pragma unroll
    for (int m = 0; m < 8; m++) {
        double x = v[m];
        for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
        if (threadIdx.x == 0) red[m][warp] = x;
    }
    __syncthreads();
    if (threadIdx.y == 0 && threadIdx.x < 8) {
        int m = threadIdx.x;
        atomicAdd(&acc[m], red[m][0] + red[m][1] + red[m][2] + red[m][3]);
    }
}

// ---------------------------------------------------------------------------
// state check (no reference counterpart: the reference lets NaN propagate,
// src/time_scheme.cpp:104-117): counts the interior cells whose values are not
// all finite or whose density or pressure is not positive.  PRIM: A is W
// (pressure read directly), else A is U (pressure from the equation of state).
template <bool PRIM>
__global__ void __launch_bounds__(128) k_check_state(const double* __restrict__ A, Box b, Consts c,
                                                     unsigned long long* __restrict__ count) {
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 4 + threadIdx.y, i = blockIdx.z;
    bool bad = false;
    if (k < b.nz && j < b.ny) {
        const long long o = b.at(i + NG, j + NG, k + NG);
        double v[5];
        bool fin = true;
#pragma unroll
        for (int q = 0; q < 5; q++) {
            v[q] = A[q * b.fstride + o];
            fin &= isfinite(v[q]);
        }
        double pr = v[1];
        if (!PRIM) {
            double w[5];
            prim_from_cons(v, c.gm1, w);
            pr = w[1];
        }
        bad = !fin || !(v[0] > 0.0) || !(pr > 0.0);
    }
    const unsigned m = __ballot_sync(0xffffffffu, bad);
    if (threadIdx.x == 0 && m) atomicAdd(count, (unsigned long long)__popc(m));
}

// ---------------------------------------------------------------------------
// host launchers

static dim3 cell_grid(const Box& b, const Planes& pl = Planes()) {  // all halo'd cells (of planes pl)
    return dim3((b.nz + 2 * NG + 31) / 32, (b.NY + 3) / 4, pl.n < 0 ? b.NX : pl.n);
}
static dim3 interior_grid(const Box& b) {
    return dim3((b.nz + 31) / 32, (b.ny + 3) / 4, b.nx);
}

void launch_step_begin(bool from_u, bool phys, double* W, double* U, double* U0, const Box& b,
                       const Consts& c, unsigned long long* slot, cudaStream_t s, Planes pl) {
    const dim3 blk(32, 4), g = cell_grid(b, pl);
    if (from_u) {
        if (phys) k_step_begin<true, true><<<g, blk, 0, s>>>(W, U, U0, b, c, slot, pl.lo);
        else k_step_begin<true, false><<<g, blk, 0, s>>>(W, U, U0, b, c, slot, pl.lo);
    } else {
        if (phys) k_step_begin<false, true><<<g, blk, 0, s>>>(W, U, U0, b, c, slot, pl.lo);
        else k_step_begin<false, false><<<g, blk, 0, s>>>(W, U, U0, b, c, slot, pl.lo);
    }
}

void launch_prim_all(double* W, const double* U, const Box& b, const Consts& c, cudaStream_t s, Planes pl) {
    k_prim_all<<<cell_grid(b, pl), dim3(32, 4), 0, s>>>(W, U, b, c, pl.lo);
}

void launch_cons_all(const double* W, double* U, const Box& b, const Consts& c, cudaStream_t s) {
    k_cons_all<<<cell_grid(b), dim3(32, 4), 0, s>>>(W, U, b, c);
}

void launch_min_dt(bool phys, const double* W, const Box& b, const Consts& c, unsigned long long* slot,
                   cudaStream_t s) {
    if (phys) k_min_dt<true><<<interior_grid(b), dim3(32, 4), 0, s>>>(W, b, c, slot);
    else k_min_dt<false><<<interior_grid(b), dim3(32, 4), 0, s>>>(W, b, c, slot);
}

void launch_fill_halo(double* W, double* U, const Box& b, const Consts& c, cudaStream_t s, double* Uhalo) {
    const long long nxe = b.nx + (c.ext_x ? 2 * NG : 0);  // slabs: y/z ghost rows of the x ghost planes too
    const long long area = std::max(std::max((long long)b.ny * b.nz, nxe * b.nz), nxe * b.ny);
    k_fill_halo<<<dim3((unsigned)((3 * area + 127) / 128), 6), 128, 0, s>>>(W, U, b, c, Uhalo);
}

void launch_fill_prim(double* W, double* U, const Box& b, const Consts& c, cudaStream_t s, double* Uhalo,
                      Planes pl) {
    k_fill_prim<<<cell_grid(b, pl), dim3(32, 4), 0, s>>>(W, U, b, c, Uhalo, pl.lo);
}

// x-planes of the face grid: all fb.n0, or the planes pl of the y- and z-faces
template <int DIR, bool CHAR, bool BORGES, bool PHYS, typename T, typename TF>
static void face_one(const double* W, const double* U, const Box& b, const Consts& c, void* F,
                     const FaceBox& fb, cudaStream_t s, bool w_only, Planes pl) {
    const int np = (DIR > 0 && pl.n >= 0) ? pl.n : fb.n0, a0 = (DIR > 0 && pl.n >= 0) ? pl.lo : 0;
    const dim3 grid((fb.n2 - (DIR == 2) + 31) / 32, (fb.n1 - (DIR == 1) + 3) / 4, np);
    const dim3 tail(((DIR == 1 ? fb.n2 : fb.n1) + 127) / 128, np);
    if constexpr (sizeof(T) == 8 && DIR > 0) {
        if (w_only) {
            k_face_flux<DIR, CHAR, BORGES, PHYS, T, TF, true><<<grid, dim3(32, 4), 0, s>>>(W, U, b, c, (TF*)F, fb, a0);
            k_face_flux_tail<DIR, CHAR, BORGES, PHYS, T, TF, true><<<tail, 128, 0, s>>>(W, U, b, c, (TF*)F, fb, a0);
            return;
        }
    }
    k_face_flux<DIR, CHAR, BORGES, PHYS, T, TF><<<grid, dim3(32, 4), 0, s>>>(W, U, b, c, (TF*)F, fb, a0);
    if constexpr (DIR > 0)
        k_face_flux_tail<DIR, CHAR, BORGES, PHYS, T, TF><<<tail, 128, 0, s>>>(W, U, b, c, (TF*)F, fb, a0);
}

template <int DIR, bool CHAR, bool BORGES, bool PHYS>
static void tail_one(const double* W, const Box& b, const Consts& c, void* F, const FaceBox& fb, cudaStream_t s,
                     Planes pl) {
    const dim3 tail(((DIR == 1 ? fb.n2 : fb.n1) + 127) / 128, pl.n < 0 ? fb.n0 : pl.n);
    k_face_flux_tail<DIR, CHAR, BORGES, PHYS, double, double, true><<<tail, 128, 0, s>>>(W, W, b, c, (double*)F, fb,
                                                                                      pl.n < 0 ? 0 : pl.lo);
}

template <int DIR>
static void tail_dispatch(bool chr, bool borges, bool phys, const double* W, const Box& b, const Consts& c, void* F,
                          const FaceBox& fb, cudaStream_t s, Planes pl) {
    if (chr) {
        if (borges) {
            if (phys) tail_one<DIR, true, true, true>(W, b, c, F, fb, s, pl);
            else tail_one<DIR, true, true, false>(W, b, c, F, fb, s, pl);
        } else {
            if (phys) tail_one<DIR, true, false, true>(W, b, c, F, fb, s, pl);
            else tail_one<DIR, true, false, false>(W, b, c, F, fb, s, pl);
        }
    } else {
        if (borges) {
            if (phys) tail_one<DIR, false, true, true>(W, b, c, F, fb, s, pl);
            else tail_one<DIR, false, true, false>(W, b, c, F, fb, s, pl);
        } else {
            if (phys) tail_one<DIR, false, false, true>(W, b, c, F, fb, s, pl);
            else tail_one<DIR, false, false, false>(W, b, c, F, fb, s, pl);
        }
    }
}

void launch_face_tail_w(int dir, bool chr, bool borges, bool phys, const double* W, const Box& b,
                        const Consts& c, void* F, const FaceBox& fb, cudaStream_t s, Planes pl) {
    if (dir == 1) tail_dispatch<1>(chr, borges, phys, W, b, c, F, fb, s, pl);
    else tail_dispatch<2>(chr, borges, phys, W, b, c, F, fb, s, pl);
}

template <int DIR, typename T, typename TF>
static void face_dispatch(bool chr, bool borges, bool phys, const double* W, const double* U,
                          const Box& b, const Consts& c, void* F, const FaceBox& fb, cudaStream_t s,
                          bool w_only, Planes pl) {
    if (chr) {
        if (borges) {
            if (phys) face_one<DIR, true, true, true, T, TF>(W, U, b, c, F, fb, s, w_only, pl);
            else face_one<DIR, true, true, false, T, TF>(W, U, b, c, F, fb, s, w_only, pl);
        } else {
            if (phys) face_one<DIR, true, false, true, T, TF>(W, U, b, c, F, fb, s, w_only, pl);
            else face_one<DIR, true, false, false, T, TF>(W, U, b, c, F, fb, s, w_only, pl);
        }
    } else {
        if (borges) {
            if (phys) face_one<DIR, false, true, true, T, TF>(W, U, b, c, F, fb, s, w_only, pl);
            else face_one<DIR, false, true, false, T, TF>(W, U, b, c, F, fb, s, w_only, pl);
        } else {
            if (phys) face_one<DIR, false, false, true, T, TF>(W, U, b, c, F, fb, s, w_only, pl);
            else face_one<DIR, false, false, false, T, TF>(W, U, b, c, F, fb, s, w_only, pl);
        }
    }
}

void launch_face_flux(int dir, bool chr, bool borges, bool phys, bool fp32, const double* W,
                      const double* U, const Box& b, const Consts& c, void* F, const FaceBox& fb,
                      cudaStream_t s, bool w_only, Planes pl) {
    if (fp32) {
        if (dir == 0) face_dispatch<0, float, float>(chr, borges, phys, W, U, b, c, F, fb, s, false, Planes());
        else if (dir == 1) face_dispatch<1, float, float>(chr, borges, phys, W, U, b, c, F, fb, s, false, Planes());
        else face_dispatch<2, float, float>(chr, borges, phys, W, U, b, c, F, fb, s, false, Planes());
    } else {
        if (dir == 0) face_dispatch<0, double, double>(chr, borges, phys, W, U, b, c, F, fb, s, w_only, pl);
        else if (dir == 1) face_dispatch<1, double, double>(chr, borges, phys, W, U, b, c, F, fb, s, w_only, pl);
        else face_dispatch<2, double, double>(chr, borges, phys, W, U, b, c, F, fb, s, w_only, pl);
    }
}

template <int MODE, int H, bool PHYS, typename TF, typename TV>
static void update_one(const UpdateArgs& a, cudaStream_t s) {
    k_update<MODE, H, PHYS, TF, TV><<<interior_grid(a.b), dim3(32, 4), 0, s>>>(
        a.W, a.U, a.U0, (const TF*)a.F[0], (const TF*)a.F[1], (const TF*)a.F[2], a.b, a.fb[0],
        a.fb[1], a.fb[2], a.c, a.flags, a.slot, a.m1, a.m2, a.mc, a.Rout, a.clock);
}

template <int MODE, bool PHYS, typename TF, typename TV>
static void update_h(int h, const UpdateArgs& a, cudaStream_t s) {
    switch (h) {
        case 0: update_one<MODE, 0, PHYS, TF, TV>(a, s); break;
        case 1: update_one<MODE, 1, PHYS, TF, TV>(a, s); break;
        case 2: update_one<MODE, 2, PHYS, TF, TV>(a, s); break;
        default: update_one<MODE, 3, PHYS, TF, TV>(a, s); break;
    }
}

template <int MODE>
static void update_mode(const UpdateArgs& a, cudaStream_t s) {
    int h = a.viscous ? a.c.order / 2 : 0;
    if (a.fp32) {
        if (a.phys) update_h<MODE, true, float, float>(h, a, s);
        else update_h<MODE, false, float, float>(h, a, s);
    } else {
        if (a.phys) update_h<MODE, true, double, double>(h, a, s);
        else update_h<MODE, false, double, double>(h, a, s);
    }
}

void launch_update(const UpdateArgs& a, cudaStream_t s) {
    if (a.mode == MODE_STAGE) update_mode<MODE_STAGE>(a, s);
    else update_mode<MODE_RHS>(a, s);
}

template <bool CHAR, bool BORGES, bool PHYS, int H>
static void xupd_one(const UpdateArgs& a, cudaStream_t s) {
    dim3 grid((a.b.nz + 31) / 32, (a.b.ny + 3) / 4, (a.b.nx + NS_XMARCH_L - 1) / NS_XMARCH_L);
    if (a.slot_next)
        k_xface_update<CHAR, BORGES, PHYS, H, true><<<grid, dim3(32, 4), 0, s>>>(
            a.W, a.U, const_cast<double*>(a.U0), a.Unext, a.Wnext, (const double*)a.F[1], (const double*)a.F[2],
            a.V, a.vs, a.b, a.fb[1], a.fb[2], a.c, a.flags, a.slot, a.slot_next, a.m1, a.m2, a.mc, a.clock);
    else
        k_xface_update<CHAR, BORGES, PHYS, H, false><<<grid, dim3(32, 4), 0, s>>>(
            a.W, a.U, const_cast<double*>(a.U0), a.Unext, a.Wnext, (const double*)a.F[1], (const double*)a.F[2],
            a.V, a.vs, a.b, a.fb[1], a.fb[2], a.c, a.flags, a.slot, nullptr, a.m1, a.m2, a.mc, a.clock);
}

template <int H, bool PHYS>
static void visc_one(const double* W, const Box& b, const Consts& c, double* V, long long vs, cudaStream_t s) {
    k_viscous<H, PHYS><<<interior_grid(b), dim3(32, 4), 0, s>>>(W, b, c, V, vs);
}

template <int H, bool PHYS>
static void visc_tma_one(const WTmaMaps& m, const double* W, const Box& b, const Consts& c, double* V, long long vs,
                         unsigned long long* err, cudaStream_t s, Planes pl) {
    constexpr size_t bytes = ViscRing<H>::smem;
    // the attribute is per device; a refusal surfaces as the launch's error
    cudaFuncSetAttribute(k_viscous_tma<H, PHYS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    // a plane range starts on a march boundary (the launcher's contract)
    const int seg0 = pl.n < 0 ? 0 : pl.lo / VISC_LX, np = pl.n < 0 ? b.nx : pl.n;
    const dim3 grid((b.nz + 31) / 32, (b.ny + 3) / 4, (np + VISC_LX - 1) / VISC_LX);
    k_viscous_tma<H, PHYS><<<grid, dim3(32, 4), bytes, s>>>(*reinterpret_cast<const CUtensorMap*>(m.map[3 + H - 1]),
                                                             W, b, c, V, vs, err, seg0);
}

void launch_viscous_tma(int h, bool phys, const WTmaMaps& m, const double* W, const Box& b, const Consts& c, double* V,
                        long long vs, unsigned long long* err, cudaStream_t s, Planes pl) {
    if (phys) {
        if (h == 1) visc_tma_one<1, true>(m, W, b, c, V, vs, err, s, pl);
        else if (h == 2) visc_tma_one<2, true>(m, W, b, c, V, vs, err, s, pl);
        else visc_tma_one<3, true>(m, W, b, c, V, vs, err, s, pl);
    } else {
        if (h == 1) visc_tma_one<1, false>(m, W, b, c, V, vs, err, s, pl);
        else if (h == 2) visc_tma_one<2, false>(m, W, b, c, V, vs, err, s, pl);
        else visc_tma_one<3, false>(m, W, b, c, V, vs, err, s, pl);
    }
}

int viscous_march_planes() { return VISC_LX; }

void launch_viscous(int h, bool phys, const double* W, const Box& b, const Consts& c, double* V,
                    long long vs, cudaStream_t s) {
    switch (h) {
        case 1: if (phys) visc_one<1, true>(W, b, c, V, vs, s); else visc_one<1, false>(W, b, c, V, vs, s); break;
        case 2: if (phys) visc_one<2, true>(W, b, c, V, vs, s); else visc_one<2, false>(W, b, c, V, vs, s); break;
        default: if (phys) visc_one<3, true>(W, b, c, V, vs, s); else visc_one<3, false>(W, b, c, V, vs, s); break;
    }
}

template <bool CHAR, bool BORGES, bool PHYS>
static void xupd_h(int h, const UpdateArgs& a, cudaStream_t s) {
    switch (h) {
        case 0: xupd_one<CHAR, BORGES, PHYS, 0>(a, s); break;
        case 1: xupd_one<CHAR, BORGES, PHYS, 1>(a, s); break;
        case 2: xupd_one<CHAR, BORGES, PHYS, 2>(a, s); break;
        default: xupd_one<CHAR, BORGES, PHYS, 3>(a, s); break;
    }
}

void launch_xface_update(bool chr, bool borges, const UpdateArgs& a, cudaStream_t s) {
    const int h = a.viscous ? a.c.order / 2 : 0;
    if (chr) {
        if (borges) { if (a.phys) xupd_h<true, true, true>(h, a, s); else xupd_h<true, true, false>(h, a, s); }
        else { if (a.phys) xupd_h<true, false, true>(h, a, s); else xupd_h<true, false, false>(h, a, s); }
    } else {
        if (borges) { if (a.phys) xupd_h<false, true, true>(h, a, s); else xupd_h<false, true, false>(h, a, s); }
        else { if (a.phys) xupd_h<false, false, true>(h, a, s); else xupd_h<false, false, false>(h, a, s); }
    }
}

void launch_check_state(const double* A, bool prim, const Box& b, const Consts& c,
                        unsigned long long* count, cudaStream_t s) {
    if (prim) k_check_state<true><<<interior_grid(b), dim3(32, 4), 0, s>>>(A, b, c, count);
    else k_check_state<false><<<interior_grid(b), dim3(32, 4), 0, s>>>(A, b, c, count);
}

void launch_slab_pack(const double* U, const Box& b, int side, double* buf, cudaStream_t s) {
    const long long n = 15LL * b.ny * b.nz;
    k_slab_pack<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(U, b, side, buf);
}
void launch_slab_unpack(double* U, const Box& b, int side, const double* buf, cudaStream_t s) {
    const long long n = 15LL * b.ny * b.nz;
    k_slab_unpack<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(U, b, side, buf);
}

void launch_aos_to_soa(const double* A, double* S, const Box& b, cudaStream_t s, Planes pl) {
    k_aos_to_soa<<<cell_grid(b, pl), dim3(32, 4), 0, s>>>(A, S, b, pl.lo);
}
void launch_soa_to_aos(const double* S, double* A, const Box& b, cudaStream_t s, Planes pl) {
    k_soa_to_aos<<<cell_grid(b, pl), dim3(32, 4), 0, s>>>(S, A, b, pl.lo);
}
void launch_diagnostics(const double* U, const Box& b, const Consts& c, double* acc, cudaStream_t s) {
    k_diagnostics<<<interior_grid(b), dim3(32, 4), 0, s>>>(U, b, c, acc);
}

}  // namespace nsb

// ---------------------------------------------------------------------------
// FMA throughput probe: the measured denominator of the compute roofline.
// Every thread runs 8 independent FMA chains (enough to cover the pipe's
// latency); the result is written only if it is NaN so the work is kept.
namespace nsb {
template <typename T>
__global__ void __launch_bounds__(256) k_fma_probe(int iters, T seed, T* sink) {
    T a[8];
#pragma unroll
    for (int c = 0; c < 8; c++) a[c] = seed + T(threadIdx.x + c);
    const T m = T(0.999999), k = T(1e-7);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int c = 0; c < 8; c++) a[c] = a[c] * m + k;
    }
    T s = a[0] + a[1] + a[2] + a[3] + a[4] + a[5] + a[6] + a[7];
    if (s != s) *sink = s;
}

cudaError_t launch_fma_probe(bool fp64, int blocks, int iters, void* sink, cudaStream_t s) {
    if (fp64)
        k_fma_probe<double><<<blocks, 256, 0, s>>>(iters, 1.0, (double*)sink);
    else
        k_fma_probe<float><<<blocks, 256, 0, s>>>(iters, 1.0f, (float*)sink);
    return cudaGetLastError();
}
}  // namespace nsb
