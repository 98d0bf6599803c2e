// ns_tma.cu -- the FP64 time step's kernels that read W through the Tensor
// Memory Accelerator (TMA): the y- and z-face fluxes from shared-memory tiles,
// the x-march over a ring of planes, and the tensor maps of W that these and
// the TMA-marched viscous kernel (ns_kernels.cu) use.
//
// The stencils of a time step read W only (U = cons(W) in registers).  A block
// of 128 threads owns 4 face rows along y x 32 faces along z of one x-plane
// and finds the 5 fields of W under those faces in shared memory: one 4D TMA
// box (z, y, x, field) of the halo'd SoA array per tile.  The kernel is
// persistent with two tile buffers: while the block computes the faces of one
// tile, the TMA engine fetches the block's next tile, so the stencil loads
// leave the warps' critical path (the per-thread kernel k_face_flux waits on
// its 30 global loads per face).  The face arithmetic is the same code
// (face_stencil_from + face_comp/face_char), so the fluxes are bit-identical.
// (A pass that formed U, the half flux and the wave speed once per cell of the
// tile in shared memory, instead of once per face through the cell, ran 2-6%
// slower on B200 at 256^3: the extra barrier and shared-memory traffic cost
// more than the 12-15% of FP64 operations it saved.)
//
// Tiles (halo'd coordinates; TMA wants the innermost start x 8 bytes and the
// box's innermost extent x 8 bytes to be multiples of 16):
//   y-faces: face (bb, kk) reads rows bb .. bb+5 at z = kk+3; box z from kk0+2
//            (even), 34 wide, rows bb0 .. bb0+8            -> 12,240 bytes
//   z-faces: face (bb, kk) reads z = kk .. kk+5 at row bb+3; box z from kk0
//            (even), 38 wide, rows bb0+3 .. bb0+6           ->  6,080 bytes
// A box that reaches past the array (last z tile of an nz that is not a
// multiple of 32) is zero-filled by the TMA unit and only feeds faces that do
// not exist.  The last face plane (j = ny or k = nz) stays with
// k_face_flux_tail, as in the per-thread path.
//
// Every mbarrier wait is bounded; a wait that runs out sets the context's error
// word (ns_synchronize then returns NS_ERR_TIMEOUT), waits, again bounded, for
// the block's copies in flight, and ends the kernel.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>

#include "ns_common.cuh"
#include "ns_eos.cuh"
#include "ns_face.cuh"
#include "ns_kernels.h"
#include "ns_tcgen05.cuh"
#include "ns_tma.cuh"

namespace nsb {

template <int DIR>
struct FaceTile;
template <>
struct FaceTile<1> {
    static constexpr int BZ = 34, BY = 9;  // box extents along z and y
    static constexpr int Z0 = 1;           // lane 0's cell along z in the box
    static constexpr int SS = BZ;          // stencil stride in the box
};
template <>
struct FaceTile<2> {
    static constexpr int BZ = 38, BY = 4;
    static constexpr int Z0 = 0;
    static constexpr int SS = 1;
};

template <int DIR>
struct FaceTileDims {
    static constexpr int QS = FaceTile<DIR>::BY * FaceTile<DIR>::BZ;  // one field of the box
    static constexpr int ELEMS = 5 * QS;
    static constexpr int STRIDE = (ELEMS + 15) / 16 * 16;  // buffers 128-byte aligned
    static constexpr uint32_t BYTES = ELEMS * 8;
};

#ifndef NS_FACE_TMA_MINB_CHAR
#define NS_FACE_TMA_MINB_CHAR 3
#endif
template <bool CHAR>
struct TmaFaceMinBlocks {
    // as the per-thread kernels: 168 / 128 registers (2 blocks of 255-register
    // characteristic-wise threads ran 5% slower on B200)
    static constexpr int value = CHAR ? NS_FACE_TMA_MINB_CHAR : 4;
};

template <int DIR, bool CHAR, bool BORGES, bool PHYS>
__global__ void __launch_bounds__(128, TmaFaceMinBlocks<CHAR>::value)
    k_face_flux_tma(const __grid_constant__ CUtensorMap map, Box b, Consts c, double* __restrict__ F, FaceBox fb,
                    unsigned long long* __restrict__ err, int x0, int xn) {
    using FT = FaceTile<DIR>;
    using TD = FaceTileDims<DIR>;
    __shared__ __align__(128) double buf[2 * TD::STRIDE];
    __shared__ __align__(8) unsigned long long full[2];
    const int lane = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + lane;
    const int nzt = (b.nz + 31) / 32, nyt = (b.ny + 3) / 4;
    const int tiles = xn * nyt * nzt;  // x-planes x0 .. x0+xn-1; the host keeps this below 2^31
    const int G = gridDim.x;
    const uint32_t bar[2] = {tc::smem_u32(&full[0]), tc::smem_u32(&full[1])};
    auto issue = [&](int t, int s) {
        const int tz = t % nzt, r = t / nzt, tyi = r % nyt, aa = x0 + r / nyt;
        const int kk0 = tz * 32, bb0 = tyi * 4;
        mbar_expect_tx(bar[s], TD::BYTES);
        tma_load_4d(tc::smem_u32(buf + s * TD::STRIDE), &map, DIR == 1 ? kk0 + 2 : kk0, DIR == 1 ? bb0 : bb0 + 3,
                    aa + NG, 0, bar[s]);
    };
    if (tid == 0) {
        tc::mbar_init(bar[0], 1);
        tc::mbar_init(bar[1], 1);
    }
    __syncthreads();
    if (tid == 0) {
        if ((int)blockIdx.x < tiles) issue(blockIdx.x, 0);
        if ((int)blockIdx.x + G < tiles) issue(blockIdx.x + G, 1);
    }
    int it = 0;
    for (int t = blockIdx.x; t < tiles; t += G, it++) {
        const int s = it & 1;
        const uint32_t par = (it >> 1) & 1;
        const bool ok = tc::mbar_wait(bar[s], par, kTilePolls);
        if (ok) {
            const int tz = t % nzt, r = t / nzt, tyi = r % nyt, aa = x0 + r / nyt;
            const int kk = tz * 32 + lane, bb = tyi * 4 + ty;
            if (kk < b.nz && bb < b.ny) {
                const double* sm = buf + s * TD::STRIDE + ty * FT::BZ + FT::Z0 + lane;
                auto ld = [&](int st, double w[5], double u[5]) {
#pragma unroll
                    for (int q = 0; q < 5; q++) w[q] = sm[q * TD::QS + st * FT::SS];
                    cons_from_prim(w, c.inv_gm1, u);
                };
                double fL[5][5], fR[5][5], wa[5], out[5];
                face_stencil_from<DIR, CHAR, PHYS, double>(ld, c, fL, fR, wa);
                if constexpr (!CHAR)
                    face_comp<double, BORGES>(fL, fR, out);
                else
                    face_char<DIR, PHYS, double, BORGES>(fL, fR, wa, c.gamma, c.inv_gm1, out);
                const long long fo = fb.at(aa, bb, kk);
#pragma unroll
                for (int q = 0; q < 5; q++) F[q * fb.fstride + fo] = out[q];
            }
        }
        // every thread is done with buffer s (and agrees on whether a wait ran out)
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicOr(err, 1ull);
                // the copies in flight: this tile's (buffer s) and the next one's (buffer s ^ 1)
                tc::mbar_wait(bar[s], par, kTilePolls);
                if (t + G < tiles) tc::mbar_wait(bar[s ^ 1], ((it + 1) >> 1) & 1, kTilePolls);
            }
            __syncthreads();
            return;
        }
        if (tid == 0 && t + 2 * G < tiles) issue(t + 2 * G, s);
    }
}

// ---------------------------------------------------------------------------
// The FP64 stage's x-march (k_xface_update's work) with its W stencil from a
// ring of 7 TMA-loaded planes: a block owns 4 rows x 32 columns and marches
// XT_LX cells along x; plane p's tile (z from k0+2, 34 wide, rows j0..j0+3,
// 5 fields; 5.4 KB) lands on its own mbarrier.  Planes i-2 .. i+3 feed the
// x-face between cells i and i+1 while plane i+4 is in flight; after the face
// the block's threads release plane i-2 together (one block barrier) and
// plane i+5 takes its slot.  The cell update's operands (U0, U, the y- and
// z-face fluxes, the viscous terms) come per thread (below), and the update
// itself is k_xface_update's.
#ifndef NS_XT_LX
#define NS_XT_LX 64
#endif
// Update operands: the characteristic-wise march stages all of them with
// cp.async while its x-face is formed; the component-wise march stages U0 and U
// only and reads the face fluxes and viscous terms at the update (8% faster
// for it, 8% slower for the characteristic-wise march, B200 at 256^3).
constexpr int XT_LX = NS_XT_LX;

template <int H, bool OPS = true, bool OPSV = true>
struct XTmaLayout {
    static constexpr int BZ = 34, BY = 4, QS = BZ * BY, ELEMS = 5 * QS;
    static constexpr int STRIDE = (ELEMS + 15) / 16 * 16;  // doubles per slot, 128-byte aligned
    static constexpr int NSLOT = 7;
    static constexpr int NOP = OPS ? (H > 0 && OPSV ? 34 : 30) : 10;
    static constexpr uint32_t TX = ELEMS * 8;
    static constexpr size_t bytes = (size_t)(NSLOT * STRIDE + (5 + NOP) * 128) * 8 + NSLOT * 8;
};

// Two blocks per SM for the characteristic-wise march (255 registers, no
// spills); three for the component-wise one (its 54 KB of shared memory allow
// them, and 170 registers hold it).
#ifndef NS_XT_MINB_CHAR
#define NS_XT_MINB_CHAR 2
#endif
#ifndef NS_XT_OPS_CHAR
#define NS_XT_OPS_CHAR 2  // characteristic-wise operands staged: 0 U0 and U, 1 and the face fluxes, 2 all
#endif
template <bool CHAR, bool BORGES, bool PHYS, int H, bool LAST>
__global__ void __launch_bounds__(128, CHAR ? NS_XT_MINB_CHAR : 3)
    k_xface_update_tma(const __grid_constant__ CUtensorMap map, const double* __restrict__ U, double* __restrict__ U0,
                       double* __restrict__ Uout, double* __restrict__ Wn, const double* __restrict__ Fy,
                       const double* __restrict__ Fz, const double* __restrict__ V, long long vs, Box b, FaceBox fy,
                       FaceBox fz, Consts c, int flags, const unsigned long long* __restrict__ slot,
                       unsigned long long* __restrict__ slot_next, double m1, double m2, double mc,
                       double* __restrict__ clock, unsigned long long* __restrict__ err, int seg0) {
    constexpr bool OPS = CHAR && NS_XT_OPS_CHAR >= 1;  // the face fluxes staged
    constexpr bool OPSV = OPS && NS_XT_OPS_CHAR >= 2;  // the viscous terms too
    using XL = XTmaLayout<H, OPS, OPSV>;
    extern __shared__ __align__(128) unsigned char xsm[];
    double* ring = reinterpret_cast<double*>(xsm);  // [NSLOT][5][BY][BZ]
    double* fprev = ring + XL::NSLOT * XL::STRIDE;   // [5][128]
    double* opnd = fprev + 5 * 128;                  // [NOP][128]
    unsigned long long* full = reinterpret_cast<unsigned long long*>(opnd + XL::NOP * 128);
    const int lane = threadIdx.x, ty = threadIdx.y, t = ty * 32 + lane;
    if (tc::smem_u32(ring) & 127u) {  // a TMA destination must be 128-byte aligned: report, touch nothing
        if (t == 0) atomicOr(err, 2ull);
        return;
    }
    const int k0 = blockIdx.x * 32, j0 = blockIdx.y * 4, x0 = (blockIdx.z + seg0) * XT_LX;
    const int k = k0 + lane, j = j0 + ty;
    const int x1 = min(x0 + XT_LX, b.nx);
    const bool live = k < b.nz && j < b.ny;
    double best = INFINITY;
    const double dt = fmin(1e10, __longlong_as_double((long long)*slot)) * c.cfl;
    const double m3 = mc * dt;
    if (clock && (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0) {
        clock[0] = dt;
        clock[1] += dt;
    }
    // plane p (x0 - 3 <= p <= x1 + 2) is the (p - x0 + 3)-th load of the block
    auto sl = [&](int p) { return (p - x0 + 3) % XL::NSLOT; };
    auto bar = [&](int p) { return tc::smem_u32(&full[sl(p)]); };
    auto par = [&](int p) { return (uint32_t)(((p - x0 + 3) / XL::NSLOT) & 1); };
    auto issue = [&](int p) {
        mbar_expect_tx(bar(p), XL::TX);
        tma_load_4d(tc::smem_u32(ring + sl(p) * XL::STRIDE), &map, k0 + 2, j0 + NG, p + NG, 0, bar(p));
    };
    if (t == 0)
        for (int q = 0; q < XL::NSLOT; q++) tc::mbar_init(tc::smem_u32(&full[q]), 1);
    __syncthreads();
    const int last = x1 + 2;  // the last plane any x-face of the block reads
    if (t == 0)
        for (int p = x0 - 3; p <= min(x0 + 3, last); p++) issue(p);
    bool ok = true;
    for (int p = x0 - 3; p <= x0 + 2; p++) ok = ok && tc::mbar_wait(bar(p), par(p), kTilePolls);
    int waited = ok ? x0 + 2 : x0 - 4;
    const int cc = ty * XL::BZ + lane + 1;
    // x-face a (between cells a-1 and a) of this thread's column: cells a-3 .. a+2
    auto xface = [&](int a, double out[5]) {
        auto ld = [&](int st, double w[5], double u[5]) {
            const double* P = ring + sl(a - 3 + st) * XL::STRIDE + cc;
#pragma unroll
            for (int q = 0; q < 5; q++) w[q] = P[q * XL::QS];
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
    for (int i = x0 - 1; i < x1; i++) {
        const long long o = b.at(i + NG, j + NG, k + NG);
        if (i >= x0 && live) {
#pragma unroll
            for (int q = 0; q < 5; q++) {
                cp_async8(&opnd[q * 128 + t], U0 + q * b.fstride + o);
                cp_async8(&opnd[(5 + q) * 128 + t], U + q * b.fstride + o);
                if constexpr (OPS) {
                    cp_async8(&opnd[(10 + q) * 128 + t], Fy + q * fy.fstride + fy.at(i, j, k));
                    cp_async8(&opnd[(15 + q) * 128 + t], Fy + q * fy.fstride + fy.at(i, j + 1, k));
                    if (convz) {
                        cp_async8(&opnd[(20 + q) * 128 + t], Fz + q * fz.fstride + fz.at(i, j, k));
                        cp_async8(&opnd[(25 + q) * 128 + t], Fz + q * fz.fstride + fz.at(i, j, k + 1));
                    }
                }
            }
            if constexpr (H > 0 && OPSV) {
                const long long e = ((long long)i * b.ny + j) * b.nz + k;
#pragma unroll
                for (int q = 0; q < 4; q++) cp_async8(&opnd[(30 + q) * 128 + t], V + q * vs + e);
            }
        }
        cp_async_commit();
        if (ok && i + 3 > waited) {
            ok = tc::mbar_wait(bar(i + 3), par(i + 3), kTilePolls);
            if (ok) waited = i + 3;
        }
        double f[5] = {0, 0, 0, 0, 0};
        if (ok && live) xface(i + 1, f);
        // every thread is done with plane i - 2 (and agrees on whether a wait ran out)
        if (__syncthreads_or(!ok)) {
            cp_async_wait_all();
            if (t == 0) {
                atomicOr(err, 1ull);
                // the loads still in flight: planes waited + 1 .. min(i + 4, last)
                for (int p = waited + 1; p <= min(i + 4, last); p++) tc::mbar_wait(bar(p), par(p), kTilePolls);
            }
            __syncthreads();
            return;
        }
        if (t == 0 && i + 5 <= last) issue(i + 5);  // into the slot of plane i - 2
        if (i < x0) {
#pragma unroll
            for (int q = 0; q < 5; q++) fprev[q * 128 + t] = f[q];
            continue;
        }
        cp_async_wait_all();
        if (!live) continue;
        // residual in k_update's order: x, y, z differences, then the viscous terms
        double r[5] = {0, 0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < 5; q++) {
            r[q] += (f[q] - fprev[q * 128 + t]) * c.inv_dx;
            fprev[q * 128 + t] = f[q];
            if constexpr (OPS) {
                r[q] += (opnd[(15 + q) * 128 + t] - opnd[(10 + q) * 128 + t]) * c.inv_dy;
                if (convz) r[q] += (opnd[(25 + q) * 128 + t] - opnd[(20 + q) * 128 + t]) * c.inv_dz;
            } else {
                r[q] += (Fy[q * fy.fstride + fy.at(i, j + 1, k)] - Fy[q * fy.fstride + fy.at(i, j, k)]) * c.inv_dy;
                if (convz)
                    r[q] += (Fz[q * fz.fstride + fz.at(i, j, k + 1)] - Fz[q * fz.fstride + fz.at(i, j, k)]) * c.inv_dz;
            }
        }
        if constexpr (H > 0) {
#pragma unroll
            for (int q = 1; q < 5; q++)
                r[q] += OPSV ? opnd[(29 + q) * 128 + t] : V[(q - 1) * vs + ((long long)i * b.ny + j) * b.nz + k];
        }
        double un[5], w[5];
#pragma unroll
        for (int q = 0; q < 5; q++) {
            un[q] = (opnd[q * 128 + t] * m1) + (opnd[(5 + q) * 128 + t] * m2) + (r[q] * m3);
            Uout[q * b.fstride + o] = un[q];
        }
        prim_from_cons(un, c.gm1, w);  // the next stage's W
        if constexpr (LAST) {
            double u0[5];
            const double d = PHYS ? local_dt_physical(w, c) : local_dt(w, c);
            if (d < best) best = d;  // NaN never lowers the minimum
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

// The bounded wait of every TMA and tensor-core kernel, on a phase that no
// arrival or transaction completes: it must give up after `polls` polls.
__global__ void k_wait_probe(unsigned polls, unsigned long long* __restrict__ out) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) tc::mbar_init(tc::smem_u32(&bar), 1);
    __syncthreads();
    const bool done = tc::mbar_wait(tc::smem_u32(&bar), 0, polls);
    if (__syncthreads_or(done)) {
        if (threadIdx.x == 0) out[0] = 0;
    } else if (threadIdx.x == 0) {
        out[0] = 1;
    }
}

cudaError_t launch_wait_probe(unsigned polls, unsigned long long* out, cudaStream_t s) {
    k_wait_probe<<<1, 32, 0, s>>>(polls, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// host side

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

bool w_tma_encode(WTmaMaps* m, const double* W, const Box& b) {
    m->ok = false;
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
    if (!enc || ((uintptr_t)W & 15) != 0) return false;
    if ((long long)b.nx * ((b.ny + 3) / 4) * ((b.nz + 31) / 32) >= (1ll << 31)) return false;
    // dimensions innermost first: z (padded row), y, x, field
    const cuuint64_t dims[4] = {(cuuint64_t)b.NZp, (cuuint64_t)b.NY, (cuuint64_t)b.NX, 5};
    const cuuint64_t strides[3] = {(cuuint64_t)b.NZp * 8, (cuuint64_t)b.NY * b.NZp * 8, (cuuint64_t)b.fstride * 8};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const cuuint32_t box1[4] = {FaceTile<1>::BZ, FaceTile<1>::BY, 1, 5};
    const cuuint32_t box2[4] = {FaceTile<2>::BZ, FaceTile<2>::BY, 1, 5};
    const cuuint32_t boxx[4] = {XTmaLayout<0>::BZ, XTmaLayout<0>::BY, 1, 5};
    const cuuint32_t boxv1[4] = {ViscTile<1>::BZ, ViscTile<1>::BY, 1, 5};
    const cuuint32_t boxv2[4] = {ViscTile<2>::BZ, ViscTile<2>::BY, 1, 5};
    const cuuint32_t boxv3[4] = {ViscTile<3>::BZ, ViscTile<3>::BY, 1, 5};
    const cuuint32_t* boxes[6] = {box1, box2, boxx, boxv1, boxv2, boxv3};
    for (int d = 0; d < 6; d++) {
        CUresult r = enc(reinterpret_cast<CUtensorMap*>(m->map[d]), CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4,
                         const_cast<double*>(W), dims, strides, boxes[d], estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return false;
    }
    m->W = W;
    m->ok = true;
    return true;
}

template <int DIR, bool CHAR, bool BORGES, bool PHYS>
static void tma_one(const WTmaMaps& m, const Box& b, const Consts& c, double* F, const FaceBox& fb, int sms,
                    unsigned long long* err, cudaStream_t s, Planes pl) {
    const int x0 = pl.n < 0 ? 0 : pl.lo, xn = pl.n < 0 ? b.nx : pl.n;
    const int tiles = xn * ((b.ny + 3) / 4) * ((b.nz + 31) / 32);
    const int grid = std::min(tiles, sms * TmaFaceMinBlocks<CHAR>::value);
    if (grid <= 0) return;
    const CUtensorMap& map = *reinterpret_cast<const CUtensorMap*>(m.map[DIR - 1]);
    k_face_flux_tma<DIR, CHAR, BORGES, PHYS><<<grid, dim3(32, 4), 0, s>>>(map, b, c, F, fb, err, x0, xn);
}

template <int DIR>
static void tma_dispatch(bool chr, bool borges, bool phys, const WTmaMaps& m, const Box& b, const Consts& c,
                         double* F, const FaceBox& fb, int sms, unsigned long long* err, cudaStream_t s, Planes pl) {
    if (chr) {
        if (borges) {
            if (phys) tma_one<DIR, true, true, true>(m, b, c, F, fb, sms, err, s, pl);
            else tma_one<DIR, true, true, false>(m, b, c, F, fb, sms, err, s, pl);
        } else {
            if (phys) tma_one<DIR, true, false, true>(m, b, c, F, fb, sms, err, s, pl);
            else tma_one<DIR, true, false, false>(m, b, c, F, fb, sms, err, s, pl);
        }
    } else {
        if (borges) {
            if (phys) tma_one<DIR, false, true, true>(m, b, c, F, fb, sms, err, s, pl);
            else tma_one<DIR, false, true, false>(m, b, c, F, fb, sms, err, s, pl);
        } else {
            if (phys) tma_one<DIR, false, false, true>(m, b, c, F, fb, sms, err, s, pl);
            else tma_one<DIR, false, false, false>(m, b, c, F, fb, sms, err, s, pl);
        }
    }
}

template <bool CHAR, bool BORGES, bool PHYS, int H, bool LAST>
static void xt_launch(const UpdateArgs& a, const WTmaMaps& m, unsigned long long* err, cudaStream_t s, Planes pl) {
    constexpr size_t bytes = XTmaLayout<H, CHAR && NS_XT_OPS_CHAR >= 1, NS_XT_OPS_CHAR >= 2>::bytes;
    auto kern = k_xface_update_tma<CHAR, BORGES, PHYS, H, LAST>;
    // the attribute is per device; a refusal surfaces as the launch's error
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    // a plane range starts on a march boundary (the launcher's contract)
    const int seg0 = pl.n < 0 ? 0 : pl.lo / XT_LX, np = pl.n < 0 ? a.b.nx : pl.n;
    const dim3 grid((a.b.nz + 31) / 32, (a.b.ny + 3) / 4, (np + XT_LX - 1) / XT_LX);
    kern<<<grid, dim3(32, 4), bytes, s>>>(*reinterpret_cast<const CUtensorMap*>(m.map[2]), a.U,
                                          const_cast<double*>(a.U0), a.Unext, a.Wnext, (const double*)a.F[1],
                                          (const double*)a.F[2], a.V, a.vs, a.b, a.fb[1], a.fb[2], a.c, a.flags,
                                          a.slot, LAST ? a.slot_next : nullptr, a.m1, a.m2, a.mc, a.clock, err, seg0);
}

template <bool CHAR, bool BORGES, bool PHYS>
static void xt_h(const UpdateArgs& a, const WTmaMaps& m, unsigned long long* err, cudaStream_t s, Planes pl) {
    const int h = a.viscous ? 1 : 0;  // the viscous terms arrive precomputed; H only sizes the operands
    if (a.slot_next) {
        if (h) xt_launch<CHAR, BORGES, PHYS, 1, true>(a, m, err, s, pl);
        else xt_launch<CHAR, BORGES, PHYS, 0, true>(a, m, err, s, pl);
    } else {
        if (h) xt_launch<CHAR, BORGES, PHYS, 1, false>(a, m, err, s, pl);
        else xt_launch<CHAR, BORGES, PHYS, 0, false>(a, m, err, s, pl);
    }
}

void launch_xface_update_tma(bool chr, bool borges, const UpdateArgs& a, const WTmaMaps& m, unsigned long long* err,
                             cudaStream_t s, Planes pl) {
    if (chr) {
        if (borges) { if (a.phys) xt_h<true, true, true>(a, m, err, s, pl); else xt_h<true, true, false>(a, m, err, s, pl); }
        else { if (a.phys) xt_h<true, false, true>(a, m, err, s, pl); else xt_h<true, false, false>(a, m, err, s, pl); }
    } else {
        if (borges) { if (a.phys) xt_h<false, true, true>(a, m, err, s, pl); else xt_h<false, true, false>(a, m, err, s, pl); }
        else { if (a.phys) xt_h<false, false, true>(a, m, err, s, pl); else xt_h<false, false, false>(a, m, err, s, pl); }
    }
}

int xmarch_planes() { return XT_LX; }

void launch_face_flux_tma(int dir, bool chr, bool borges, bool phys, const WTmaMaps& m, const double* W,
                          const Box& b, const Consts& c, void* F, const FaceBox& fb, int sms,
                          unsigned long long* err, cudaStream_t s, Planes pl) {
    if (dir == 1) tma_dispatch<1>(chr, borges, phys, m, b, c, (double*)F, fb, sms, err, s, pl);
    else tma_dispatch<2>(chr, borges, phys, m, b, c, (double*)F, fb, sms, err, s, pl);
    launch_face_tail_w(dir, chr, borges, phys, W, b, c, F, fb, s, pl);
}

}  // namespace nsb
