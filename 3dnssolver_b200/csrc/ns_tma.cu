// ns_tma.cu -- y- and z-face fluxes of the FP64 time steps from shared-memory
// tiles that the Tensor Memory Accelerator (TMA) loads, and the tensor maps of
// W that this kernel and the TMA-marched viscous kernel (ns_kernels.cu) use.
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

template <bool CHAR>
struct TmaFaceMinBlocks {
    // as the per-thread kernels: 168 / 128 registers (2 blocks of 255-register
    // characteristic-wise threads ran 5% slower on B200)
    static constexpr int value = CHAR ? 3 : 4;
};

template <int DIR, bool CHAR, bool BORGES, bool PHYS>
__global__ void __launch_bounds__(128, TmaFaceMinBlocks<CHAR>::value)
    k_face_flux_tma(const __grid_constant__ CUtensorMap map, Box b, Consts c, double* __restrict__ F, FaceBox fb,
                    unsigned long long* __restrict__ err) {
    using FT = FaceTile<DIR>;
    using TD = FaceTileDims<DIR>;
    __shared__ __align__(128) double buf[2 * TD::STRIDE];
    __shared__ __align__(8) unsigned long long full[2];
    const int lane = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + lane;
    const int nzt = (b.nz + 31) / 32, nyt = (b.ny + 3) / 4;
    const int tiles = b.nx * nyt * nzt;  // the host keeps this below 2^31
    const int G = gridDim.x;
    const uint32_t bar[2] = {tc::smem_u32(&full[0]), tc::smem_u32(&full[1])};
    auto issue = [&](int t, int s) {
        const int tz = t % nzt, r = t / nzt, tyi = r % nyt, aa = r / nyt;
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
            const int tz = t % nzt, r = t / nzt, tyi = r % nyt, aa = r / nyt;
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
    const cuuint32_t boxv[4] = {VISC_TMA_BZ, VISC_TMA_BY, 1, 5};
    const cuuint32_t* boxes[3] = {box1, box2, boxv};
    for (int d = 0; d < 3; d++) {
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
                    unsigned long long* err, cudaStream_t s) {
    const int tiles = b.nx * ((b.ny + 3) / 4) * ((b.nz + 31) / 32);
    const int grid = std::min(tiles, sms * TmaFaceMinBlocks<CHAR>::value);
    const CUtensorMap& map = *reinterpret_cast<const CUtensorMap*>(m.map[DIR - 1]);
    k_face_flux_tma<DIR, CHAR, BORGES, PHYS><<<grid, dim3(32, 4), 0, s>>>(map, b, c, F, fb, err);
}

template <int DIR>
static void tma_dispatch(bool chr, bool borges, bool phys, const WTmaMaps& m, const Box& b, const Consts& c,
                         double* F, const FaceBox& fb, int sms, unsigned long long* err, cudaStream_t s) {
    if (chr) {
        if (borges) {
            if (phys) tma_one<DIR, true, true, true>(m, b, c, F, fb, sms, err, s);
            else tma_one<DIR, true, true, false>(m, b, c, F, fb, sms, err, s);
        } else {
            if (phys) tma_one<DIR, true, false, true>(m, b, c, F, fb, sms, err, s);
            else tma_one<DIR, true, false, false>(m, b, c, F, fb, sms, err, s);
        }
    } else {
        if (borges) {
            if (phys) tma_one<DIR, false, true, true>(m, b, c, F, fb, sms, err, s);
            else tma_one<DIR, false, true, false>(m, b, c, F, fb, sms, err, s);
        } else {
            if (phys) tma_one<DIR, false, false, true>(m, b, c, F, fb, sms, err, s);
            else tma_one<DIR, false, false, false>(m, b, c, F, fb, sms, err, s);
        }
    }
}

void launch_face_flux_tma(int dir, bool chr, bool borges, bool phys, const WTmaMaps& m, const double* W,
                          const Box& b, const Consts& c, void* F, const FaceBox& fb, int sms,
                          unsigned long long* err, cudaStream_t s) {
    if (dir == 1) tma_dispatch<1>(chr, borges, phys, m, b, c, (double*)F, fb, sms, err, s);
    else tma_dispatch<2>(chr, borges, phys, m, b, c, (double*)F, fb, sms, err, s);
    launch_face_tail_w(dir, chr, borges, phys, W, b, c, F, fb, s);
}

}  // namespace nsb
