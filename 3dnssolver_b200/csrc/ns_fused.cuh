// ns_fused.cuh -- one kernel per SSP-RK3 stage (FP32 form, reference or
// physical semantics).  The kernel template lives here; ns_fused_ref.cu and
// ns_fused_phys.cu instantiate it per semantics (parallel builds) and
// ns_fused.cu dispatches.
//
// A block owns a TY x TZ column of cells and marches along x.  Every plane it
// touches is loaded once with 3 ghost rows and columns, folding each axis by
// its boundary condition (periodic wrap or Neumann clamp: the single-GPU form
// of Domain::apply_boundary_conditions + Communicator::communicate,
// src/domain.cpp:18-28, src/communicator.cpp:6-143), and kept as W = prim(U)
// (src/eq_of_state.cpp:61-87) in a shared-memory ring of 7 planes.  For each
// cell it forms the face fluxes along x (carried from cell to cell in
// registers), y and z, accumulates (f(+) - f(-))/d in the reference's order
// (Weno5::compute_residual, weno-5.cpp:39-73), adds the centered viscous terms
// from the ring, and writes U_out = U0 m1 + U_in m2 + R mc dt
// (TimeScheme::substep, time_scheme.cpp:72-96).  U_in and U_out are different
// buffers: neighbouring blocks read U_in's cells as their ghost layers.
//
// The third stage also takes the next step's start: W = prim(U_out) for the
// CFL minimum (time_scheme.cpp:69, 98-136) and U0 = cons(W) (the W -> U
// round trip of time_scheme.cpp:124), so a step is three launches.
//
// The Lax-Friedrichs split uses U = cons(W) of the ring's W; it differs from
// the stage's U by rounding only.
//
// PHYS (physical semantics, no reference counterpart): local Lax-Friedrichs
// speed and the textbook eigensystem in the faces (ns_face_f32x2.cuh), the full
// 3D viscous stress and heat flux from the ring (march_viscous_physical) and
// the multi-dimensional CFL bound in the third stage.
#pragma once
#include <cuda_runtime.h>

#include "ns_common.cuh"
#include "ns_eos.cuh"
#include "ns_face.cuh"
#include "ns_face_f32x2.cuh"
#include "ns_kernels.h"
#include "ns_viscous.cuh"

namespace nsb {

// ---------------------------------------------------------------------------
// A block marches LX cells along x over a TY x TZ column: 2.2 plane loads per
// cell (a 3D box tile with the same shared memory needed 7.4 and ran 20%
// slower on B200), x-face fluxes carried in registers, y- and z-faces of the
// current plane through small shared face buffers.

// TY x TZ = 8 x 32 cells per plane, one per thread.  A 7-row tile (one round
// per face pass instead of two for the 288 y- and 264 z-faces) measured the
// same on B200 (+2.6% component-wise, -3% characteristic), so the plane of 8
// rows stays; NS_MARCH_TY selects it at build time.
#ifndef NS_MARCH_TY
#define NS_MARCH_TY 8
#endif
// cells a block marches along x: 64 ran 2.2% faster than 32 for the
// characteristic-wise stage on B200 at 256^3 and 0.5% slower for the
// component-wise one
template <bool CHAR>
struct MarchLen {
    static constexpr int value = CHAR ? 64 : 32;
};
//
// Plane i reads planes i-2..i+3 (x-faces) and i-H..i+H (viscous terms).  With
// H <= 1 ("lean") the ring holds 6 planes and the y/z face buffers alternate
// between planes, so a plane needs two block barriers instead of three: the
// next plane's conversion overwrites plane i-2, whose last reader (the x-faces)
// finished before this plane's second barrier.
//
// The FP32 form runs here; the FP64 form runs the face kernels and the x-face
// march of ns_kernels.cu.  An FP64 variant of this kernel on an 8 x 16 column
// (128 threads, 109 KB, two blocks of 252 registers per SM) reproduced the FP64
// path's results exactly but ran 1.25-1.56x slower on B200 (Taylor-Green and
// shear layer at 256^3): with 8 warps per SM and the plane barriers, the FP64
// pipe idles; the separate face kernels keep it 62-67% busy at 12 warps.
template <typename T, int H = 1>
struct MarchTile {
    static_assert(sizeof(T) == 4, "the fused stage serves the FP32 form");
    static constexpr int TY = NS_MARCH_TY, TZ = 32;
    static constexpr int FT = TY * TZ;  // threads per block, one per cell of the column
    static constexpr int PY = TY + 6, PZ = TZ + 6, NP = PY * PZ;
    static constexpr bool LEAN = H <= 1;
    static constexpr int RING = LEAN ? 6 : 7;
    static constexpr int NBUF = LEAN ? 2 : 1;
    static constexpr int NFY = (TY + 1) * TZ, NFZ = TY * (TZ + 1);
    static constexpr int MINB = 2;
    // ring, y/z face buffers, and the FP64 conserved state of the plane in flight
    static constexpr size_t smem = (size_t)RING * 5 * NP * sizeof(T) +
                                   (size_t)NBUF * 5 * (NFY + NFZ) * sizeof(T) + (size_t)5 * NP * sizeof(double);
};


// Thread index rotated so that warp w handles items 0..31 of every round of a
// pass: the partial last round of each pass (plane loads, y-faces, z-faces)
// then falls to a different warp instead of piling up on warp 0 before the
// same barrier.
template <int FT>
__device__ __forceinline__ int rotated(int tid, int w) { return (tid + FT - (32 * w) % FT) % FT; }

template <int RING>
__device__ __forceinline__ int ring_slot(int i, int x0) {
    return (i - x0 + 3) % RING;  // i >= x0 - 3
}

// one face from a 6-cell stencil in a shared array with stride `step`
template <int DIR, bool CHAR, bool BORGES, bool PHYS, typename T>
__device__ __forceinline__ void march_face(const T* const* planes, int c0, int step, int fs, const Consts& c,
                                           T out[5]) {
    face_f32x2<DIR, CHAR, BORGES, PHYS>(planes, c0, step, fs, T(c.gamma), T(c.inv_gm1), out);
}


// centered viscous terms of the cell at plane i, in-plane index cc, from the
// ring (reference semantics): mixed derivatives differentiate first
// derivatives that are zero outside the interior along a non-periodic axis
// (centered_diffusion.cpp:22-24)
template <int H, typename T, typename PlaneFn>
__device__ __forceinline__ void march_viscous(PlaneFn plane, int i, int cc, const Consts& c, int nx,
                                              int ny, int gi, int gj, T r[5]) {
    using M = MarchTile<T>;
    const int sy = M::PZ, fs = M::NP;
    T cx1[2 * H + 1], cy1[2 * H + 1], cxx[2 * H + 1], cyy[2 * H + 1];
#pragma unroll
    for (int t = 0; t <= 2 * H; t++) {
        cx1[t] = T(c.df[3 - H + t] * c.inv_dx);
        cy1[t] = T(c.df[3 - H + t] * c.inv_dy);
        cxx[t] = T(c.ddf[3 - H + t] * c.inv_dx * c.inv_dx);
        cyy[t] = T(c.ddf[3 - H + t] * c.inv_dy * c.inv_dy);
    }
    const T* P[2 * H + 1];
#pragma unroll
    for (int t = 0; t <= 2 * H; t++) P[t] = plane(i + t - H);
    T Dx[4], Dy[4], Dxx[4], Dyy[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        T a1 = 0, b1 = 0, a2 = 0, b2 = 0;
#pragma unroll
        for (int t = 0; t <= 2 * H; t++) {
            T wx = P[t][q * fs + cc];
            T wy = P[H][q * fs + cc + (t - H) * sy];
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
                    if (t != H) dx += P[t][q * fs + cc + (s - H) * sy] * cx1[t];
                sxy += dx * cy1[s];
            }
            int ii = gi + s - H;
            if (x_inside(ii, nx, c)) {
                T dy = 0;
#pragma unroll
                for (int t = 0; t <= 2 * H; t++)
                    if (t != H) dy += P[s][q * fs + cc + (t - H) * sy] * cy1[t];
                syx += dy * cx1[s];
            }
        }
        Dxy[v] = sxy; Dyx[v] = syx;
    }
    viscous_reference_terms<T>(Dx, Dy, Dxx, Dyy, Dxy, Dyx, P[H][2 * fs + cc], P[H][3 * fs + cc],
                               P[H][1 * fs + cc], P[H][cc], c, r);
}

// centered viscous terms of the cell at plane i, in-plane index cc, from the
// ring, physical semantics (no reference counterpart): the full 3D stress and
// heat flux with constant mu, the same terms as viscous_physical in
// ns_kernels.cu.  The ring's cells are boundary-folded along every axis, so
// mixed derivatives read folded edge and corner cells like viscous_physical.
template <int H, typename T, typename PlaneFn>
__device__ __forceinline__ void march_viscous_physical(PlaneFn plane, int i, int cc, const Consts& c,
                                                       T r[5]) {
    using M = MarchTile<T>;
    const int sy = M::PZ, fs = M::NP;
    const int nd = c.dim == 3 ? 3 : 2;
    const T* P[2 * H + 1];
#pragma unroll
    for (int t = 0; t <= 2 * H; t++) P[t] = plane(i + t - H);
    const double inv[3] = {c.inv_dx, c.inv_dy, c.inv_dz};
    T c1[3][2 * H + 1], c2[3][2 * H + 1];
#pragma unroll
    for (int ax = 0; ax < 3; ax++)
#pragma unroll
        for (int t = 0; t <= 2 * H; t++) {
            c1[ax][t] = T(c.df[3 - H + t] * inv[ax]);
            c2[ax][t] = T(c.ddf[3 - H + t] * inv[ax] * inv[ax]);
        }
    // field q of the cell offset by (ox planes, oy rows, oz columns)
    auto at = [&](int q, int ox, int oy, int oz) -> T { return P[H + ox][q * fs + cc + oy * sy + oz]; };
    T gu[3][3] = {}, lap[3] = {}, gdiv[3] = {}, lapT = 0;
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
        if (ax >= nd) continue;
#pragma unroll
        for (int t = 0; t <= 2 * H; t++) {
            const int ox = ax == 0 ? t - H : 0, oy = ax == 1 ? t - H : 0, oz = ax == 2 ? t - H : 0;
            const T Tt = at(1, ox, oy, oz) / at(0, ox, oy, oz);
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const T va = at(2 + a, ox, oy, oz);
                gu[a][ax] += va * c1[ax][t];
                lap[a] += va * c2[ax][t];
                if (a == ax) gdiv[a] += va * c2[ax][t];
            }
            lapT += Tt * c2[ax][t];
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int bx = 0; bx < 3; bx++) {
            if (a == bx || a >= nd || bx >= nd) continue;
            T acc = 0;
#pragma unroll
            for (int s = 0; s <= 2 * H; s++)
#pragma unroll
                for (int t = 0; t <= 2 * H; t++) {
                    int o[3] = {0, 0, 0};
                    o[a] += s - H;
                    o[bx] += t - H;
                    acc += at(2 + bx, o[0], o[1], o[2]) * c1[a][s] * c1[bx][t];
                }
            gdiv[a] += acc;
        }
    const T mu = T(c.mu), lamb = T(c.lamb);
    const T uv[3] = {at(2, 0, 0, 0), at(3, 0, 0, 0), at(4, 0, 0, 0)};
    const T div = gu[0][0] + gu[1][1] + gu[2][2];
    T work = 0, diss = 0, mom[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        mom[a] = mu * lap[a] + (mu + lamb) * gdiv[a];
        work += uv[a] * mom[a];
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int bx = 0; bx < 3; bx++) {
            const T tab = mu * (gu[a][bx] + gu[bx][a]) + (a == bx ? lamb * div : T(0));
            diss += tab * gu[a][bx];
        }
    r[2] -= mom[0];
    r[3] -= mom[1];
    r[4] -= mom[2];
    r[1] -= work + diss + T(c.heat) * mu * lapT;
}

template <typename T, bool CHAR, bool BORGES, int H, bool LAST, bool PHYS>
__global__ void __launch_bounds__(MarchTile<T, H>::FT, MarchTile<T, H>::MINB)
    k_stage_march(const double* __restrict__ Uin, double* U0, double* __restrict__ Uout, Box b,
                  Consts c, int conv_dims, double m1, double m2, double mc,
                  const unsigned long long* __restrict__ slot, unsigned long long* slot_next,
                  double* clock, const unsigned char* __restrict__ skip) {
    using M = MarchTile<T, H>;
    constexpr int FT = M::FT;
    static_assert(M::NFY <= 2 * FT && M::NFZ <= 2 * FT, "a face pass takes at most two rounds");
    extern __shared__ __align__(16) unsigned char smem[];
    T* ring = reinterpret_cast<T*>(smem);        // [RING][5][NP]
    T* FYb = ring + M::RING * 5 * M::NP;         // [NBUF][5][NFY]
    T* FZb = FYb + M::NBUF * 5 * M::NFY;         // [NBUF][5][NFZ]
    double* S = reinterpret_cast<double*>(FZb + M::NBUF * 5 * M::NFZ);  // [5][NP] U_in of the plane in flight
    const int tid = threadIdx.x, ty = tid / M::TZ, tz = tid % M::TZ;
    constexpr int LX = MarchLen<CHAR>::value;
    const int k0 = blockIdx.x * M::TZ, j0 = blockIdx.y * M::TY, x0 = blockIdx.z * LX;
    const int x1 = min(x0 + LX, b.nx);
    auto plane = [&](int i) { return ring + ring_slot<M::RING>(i, x0) * 5 * M::NP; };
    // U_in of plane i at folded positions, into S without waiting (each thread
    // later converts exactly the elements it copied, so S needs no barrier)
    auto issue_plane = [&](int i) {
        const int gi = fold_x(i, b.nx, c);
        for (int e = rotated<FT>(tid, 5); e < M::NP; e += FT) {
            int py = e / M::PZ, pz = e % M::PZ;
            int gj = fold(j0 - 3 + py, b.ny, c.periodic[1]);
            int gk = fold(k0 - 3 + pz, b.nz, c.periodic[2]);
            long long o = b.at(gi + NG, gj + NG, gk + NG);
#pragma unroll
            for (int q = 0; q < 5; q++) cp_async8(S + q * M::NP + e, Uin + q * b.fstride + o);
        }
        cp_async_commit();
    };
    // W = prim(U_in) of the plane in S into plane i's ring slot
    auto convert_plane = [&](int i) {
        cp_async_wait_all();
        T* P = plane(i);
        for (int e = rotated<FT>(tid, 5); e < M::NP; e += FT) {
            if constexpr (sizeof(T) == 4) {
                // the FP32 form's W in FP32 arithmetic from the FP64 state
                float u[5];
#pragma unroll
                for (int q = 0; q < 5; q++) u[q] = float(S[q * M::NP + e]);
                const float ir = __fdividef(1.f, u[0]);
                const float vx = u[2] * ir, vy = u[3] * ir, vz = u[4] * ir;
                P[e] = u[0];
                P[M::NP + e] = float(c.gm1) * (u[1] - 0.5f * u[0] * (vx * vx + vy * vy + vz * vz));
                P[2 * M::NP + e] = vx;
                P[3 * M::NP + e] = vy;
                P[4 * M::NP + e] = vz;
            } else {
                double u[5], w[5];
#pragma unroll
                for (int q = 0; q < 5; q++) u[q] = S[q * M::NP + e];
                prim_from_cons(u, c.gm1, w);
#pragma unroll
                for (int q = 0; q < 5; q++) P[q * M::NP + e] = T(w[q]);
            }
        }
    };
    auto load_plane = [&](int i) {
        issue_plane(i);
        convert_plane(i);
    };
    // x-face of this thread's column between cells i and i+1 (stencil i-2..i+3)
    const int ccol = (ty + 3) * M::PZ + (tz + 3);
    auto xface = [&](int i, T out[5]) {
        const T* P[6];
#pragma unroll
        for (int s = 0; s < 6; s++) P[s] = plane(i - 2 + s);
        march_face<0, CHAR, BORGES, PHYS, T>(P, ccol, 0, M::NP, c, out);
    };
    const int gj = j0 + ty, gk = k0 + tz;
    const bool row = ty < M::TY;  // the eighth warp only helps with the y- and z-faces
    const bool own = row && gj < b.ny && gk < b.nz;
    for (int i = x0 - 3; i < x0 + 3; i++) load_plane(i);
    issue_plane(x0 + 3);
    __syncthreads();
    T fxl[5] = {0, 0, 0, 0, 0}, fxr[5];
    if (conv_dims > 0 && row) xface(x0 - 1, fxl);
    if constexpr (M::LEAN) __syncthreads();  // plane x0+3 takes the slot of plane x0-3
    const double dt = fmin(1e10, __longlong_as_double((long long)*slot)) * c.cfl;
    const double m3 = mc * dt;
    if (clock && (blockIdx.x | blockIdx.y | blockIdx.z | tid) == 0) {
        clock[0] = dt;
        clock[1] += dt;
    }
    double best = INFINITY;
    for (int i = x0; i < x1; i++) {
        convert_plane(i + 3);
        __syncthreads();
        if (i + 1 < x1) issue_plane(i + 4);  // in flight during this plane's faces and update
        const T* Pi = plane(i);
        T* FY = FYb + (M::NBUF == 2 ? ((i - x0) & 1) : 0) * 5 * M::NFY;
        T* FZ = FZb + (M::NBUF == 2 ? ((i - x0) & 1) : 0) * 5 * M::NFZ;
        if (conv_dims > 0) {
            if (row) xface(i, fxr);
            // y-faces of plane i: between rows fb-1 and fb, stencil rows fb..fb+5 of the plane
            for (int e = rotated<FT>(tid, 7); e < M::NFY; e += FT) {
                int fb = e / M::TZ, cz = e % M::TZ;
                const T* P[6] = {Pi, Pi, Pi, Pi, Pi, Pi};
                T out[5];
                march_face<1, CHAR, BORGES, PHYS, T>(P, fb * M::PZ + cz + 3, M::PZ, M::NP, c, out);
#pragma unroll
                for (int q = 0; q < 5; q++) FY[q * M::NFY + e] = out[q];
            }
            if (conv_dims == 3) {
                for (int e = rotated<FT>(tid, 6); e < M::NFZ; e += FT) {
                    int ry = e / (M::TZ + 1), fc = e % (M::TZ + 1);
                    const T* P[6] = {Pi, Pi, Pi, Pi, Pi, Pi};
                    T out[5];
                    march_face<2, CHAR, BORGES, PHYS, T>(P, (ry + 3) * M::PZ + fc, 1, M::NP, c, out);
#pragma unroll
                    for (int q = 0; q < 5; q++) FZ[q * M::NFZ + e] = out[q];
                }
            }
        }
        __syncthreads();
        if (own) {
            const long long o = b.at(i + NG, gj + NG, gk + NG);
            double u0[5], ui[5];
#pragma unroll
            for (int q = 0; q < 5; q++) {  // issued before the viscous terms hide their latency
                u0[q] = U0[q * b.fstride + o];
                ui[q] = Uin[q * b.fstride + o];
            }
            double r[5] = {0, 0, 0, 0, 0};
            if (conv_dims > 0) {
#pragma unroll
                for (int q = 0; q < 5; q++) {
                    r[q] += (double(fxr[q]) - double(fxl[q])) * c.inv_dx;
                    r[q] += (double(FY[q * M::NFY + (ty + 1) * M::TZ + tz]) -
                             double(FY[q * M::NFY + ty * M::TZ + tz])) * c.inv_dy;
                    if (conv_dims == 3)
                        r[q] += (double(FZ[q * M::NFZ + ty * (M::TZ + 1) + tz + 1]) -
                                 double(FZ[q * M::NFZ + ty * (M::TZ + 1) + tz])) * c.inv_dz;
                }
            }
            if constexpr (H > 0) {
                T rv[5] = {0, 0, 0, 0, 0};
                if constexpr (PHYS)
                    march_viscous_physical<H, T>(plane, i, ccol, c, rv);
                else
                    march_viscous<H, T>(plane, i, ccol, c, b.nx, b.ny, i, gj, rv);
#pragma unroll
                for (int q = 1; q < 5; q++) r[q] += double(rv[q]);
            }
            double un[5];
#pragma unroll
            for (int q = 0; q < 5; q++) {
                un[q] = (u0[q] * m1) + (ui[q] * m2) + (r[q] * m3);
                Uout[q * b.fstride + o] = un[q];
            }
            // the sensor's correction pass forms the next step's start of the cells it corrects
            if (LAST && !(skip && skip[((long long)i * b.ny + gj) * b.nz + gk])) {
                double w[5], un0[5];
                prim_from_cons(un, c.gm1, w);
                double d = PHYS ? local_dt_physical(w, c) : local_dt(w, c);
                if (d < best) best = d;
                cons_from_prim(w, c.inv_gm1, un0);
#pragma unroll
                for (int q = 0; q < 5; q++) U0[q * b.fstride + o] = un0[q];
            }
        }
#pragma unroll
        for (int q = 0; q < 5; q++) fxl[q] = fxr[q];
        if constexpr (!M::LEAN) __syncthreads();
    }
    if constexpr (LAST) block_min_to(best, slot_next);
}

template <typename T, bool CHAR, bool BORGES, int H, bool LAST, bool PHYS>
static cudaError_t fused_one(const FusedArgs& a, cudaStream_t s) {
    using M = MarchTile<T, H>;
    auto kern = k_stage_march<T, CHAR, BORGES, H, LAST, PHYS>;
    // the attribute is per device; setting it on every launch keeps multi-device use correct
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)M::smem);
    if (e != cudaSuccess) return e;
    constexpr int LX = MarchLen<CHAR>::value;
    dim3 grid((a.b.nz + M::TZ - 1) / M::TZ, (a.b.ny + M::TY - 1) / M::TY, (a.b.nx + LX - 1) / LX);
    kern<<<grid, M::FT, M::smem, s>>>(a.Uin, a.U0, a.Uout, a.b, a.c, a.conv_dims, a.m1, a.m2, a.mc, a.slot,
                                   a.slot_next, a.clock, a.skip);
    return cudaGetLastError();
}

template <typename T, bool PHYS, bool CHAR, bool BORGES, bool LAST>
static cudaError_t fused_h(const FusedArgs& a, cudaStream_t s) {
    switch (a.visc_h) {
        case 0: return fused_one<T, CHAR, BORGES, 0, LAST, PHYS>(a, s);
        case 1: return fused_one<T, CHAR, BORGES, 1, LAST, PHYS>(a, s);
        case 2: return fused_one<T, CHAR, BORGES, 2, LAST, PHYS>(a, s);
        default: return fused_one<T, CHAR, BORGES, 3, LAST, PHYS>(a, s);
    }
}

// One fused FP32 stage of the given semantics (instantiated per semantics in
// ns_fused_{ref,phys}.cu).
template <typename T, bool PHYS>
cudaError_t fused_launch(const FusedArgs& a, cudaStream_t s) {
    if (!a.fp32) return cudaErrorInvalidValue;
    if (a.chr) {
        if (a.borges)
            return a.last ? fused_h<T, PHYS, true, true, true>(a, s) : fused_h<T, PHYS, true, true, false>(a, s);
        return a.last ? fused_h<T, PHYS, true, false, true>(a, s) : fused_h<T, PHYS, true, false, false>(a, s);
    }
    if (a.borges) return a.last ? fused_h<T, PHYS, false, true, true>(a, s) : fused_h<T, PHYS, false, true, false>(a, s);
    return a.last ? fused_h<T, PHYS, false, false, true>(a, s) : fused_h<T, PHYS, false, false, false>(a, s);
}

extern template cudaError_t fused_launch<float, false>(const FusedArgs& a, cudaStream_t s);
extern template cudaError_t fused_launch<float, true>(const FusedArgs& a, cudaStream_t s);

}  // namespace nsb
