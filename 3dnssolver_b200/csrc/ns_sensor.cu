// ns_sensor.cu -- learned troubled-face sensor (no reference counterpart).
//
// A small MLP (21 -> 32 -> 32 -> 1, GELU in its tanh form) looks at the stencil of a face and
// predicts whether the characteristic-wise WENO-5 flux differs from the
// component-wise one by more than a relative threshold.  The gated FP32 form
// computes the cheap component-wise flux on every face, evaluates the MLP on
// the tensor cores, and recomputes the characteristic-wise flux only on the
// faces it flags.
//
// Tensor cores: mma.sync.m16n8k16 with BF16 operands and FP32 accumulation;
// one warp owns 32 faces (two 16-row tiles), hidden width 32 (four 8-column
// tiles), input width 32 (21 features + zero padding, two 16-deep k steps).
// The 32x32 layers are too narrow for tcgen05/TMEM to pay off: the MLP is a
// few percent of a gated face's cost either way.
//
// Features of a face between cells a and a+1 (stencil a-2..a+3): for X in
// (rho, p, u_n) the six values centred on their mean and scaled by their
// largest deviation plus 1e-3 of a reference scale (18 values), and the three
// Jiang-Shu smoothness indicators of rho on a-2..a+2 normalised by their sum
// (3 values).  Labels: |f_char - f_comp|_2 / (|f_char|_2 + 1e-12) > threshold,
// both fluxes in FP64 with the reference semantics.
//
// Parameter layout (floats): W1[32][32] (out, in; in >= 21 unused), b1[32],
// W2[32][32] (out, in), b2[32], w3[32], b3.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "ns_common.cuh"
#include "ns_eos.cuh"
#include "ns_face.cuh"
#include "ns_sensor.h"
#include "ns_tcgen05.cuh"

namespace nsb {

constexpr int SF = NS_SENSOR_FEATURES;  // 21
constexpr int SH = 32;                  // hidden width
constexpr int SP = NS_SENSOR_NPARAMS;   // 2145
constexpr int OFF_W1 = 0, OFF_B1 = 1024, OFF_W2 = 1056, OFF_B2 = 2080, OFF_W3 = 2112, OFF_B3 = 2144;
constexpr int XS = 40;  // bf16 row stride of the smem tiles (conflict-free fragment loads)

// The per-step flags run the network on the 5th-generation tensor cores
// (tcgen05.mma, TMEM accumulators); training and ns_sensor_predict use the
// warp-level mma.sync tiles below.  A warp-level mma.sync variant of the flag
// kernel measured within 3% of the tcgen05 one on B200: the flag pass is bound
// by its feature loads and GELU, not by the two small matrix products.

// ---------------------------------------------------------------------------
// tensor-core building blocks

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ uint32_t pack_bf16_raw(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// D = A(16x16, row) * B(16x8, col) + D; BF16 operands, FP32 accumulators
__device__ __forceinline__ void mma16816(float d[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// GELU in its tanh form, 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))) (Hendrycks &
// Gimpel 2016), on the special-function unit's tanh (tanh.approx.f32, ~2^-11 relative)
__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float gelu(float x) {
    const float k0 = 0.7978845608028654f, k1 = 0.044715f;
    return 0.5f * x * (1.0f + tanh_fast(k0 * (x + k1 * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float k0 = 0.7978845608028654f, k1 = 0.044715f;
    float t = tanh_fast(k0 * (x + k1 * x * x * x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * k0 * (1.0f + 3.0f * k1 * x * x);
}

// smem copy of the network: bf16 weight tiles (row = output unit), FP32 vectors
struct MlpSmem {
    __nv_bfloat16 W1[SH * XS];
    __nv_bfloat16 W2[SH * XS];
    __nv_bfloat16 W2T[SH * XS];  // backward only
    float b1[SH], b2[SH], w3[SH], b3;
};

__device__ void mlp_load(MlpSmem& m, const float* __restrict__ w, bool transpose) {
    for (int e = threadIdx.x + threadIdx.y * blockDim.x; e < SH * XS; e += blockDim.x * blockDim.y) {
        int r = e / XS, col = e % XS;
        m.W1[e] = __float2bfloat16(col < SF ? w[OFF_W1 + r * 32 + col] : 0.f);
        m.W2[e] = __float2bfloat16(col < SH ? w[OFF_W2 + r * 32 + col] : 0.f);
        if (transpose) m.W2T[e] = __float2bfloat16(col < SH ? w[OFF_W2 + col * 32 + r] : 0.f);
    }
    for (int e = threadIdx.x + threadIdx.y * blockDim.x; e < SH; e += blockDim.x * blockDim.y) {
        m.b1[e] = w[OFF_B1 + e];
        m.b2[e] = w[OFF_B2 + e];
        m.w3[e] = w[OFF_W3 + e];
    }
    if (threadIdx.x + threadIdx.y == 0) m.b3 = w[OFF_B3];
}

// B fragment of a [n][k] row-major bf16 tile: k = 16 kt + 2q (+8), n = 8 nt + g
__device__ __forceinline__ void bfrag(const __nv_bfloat16* T, int nt, int kt, int g, int q, uint32_t b[2]) {
    const __nv_bfloat16* p = T + (8 * nt + g) * XS + 16 * kt + 2 * q;
    b[0] = *reinterpret_cast<const uint32_t*>(p);
    b[1] = *reinterpret_cast<const uint32_t*>(p + 8);
}

// A fragment of a [m][k] row-major bf16 tile (rows 16 mt..)
__device__ __forceinline__ void afrag(const __nv_bfloat16* T, int mt, int kt, int g, int q, uint32_t a[4]) {
    const __nv_bfloat16* p = T + (16 * mt + g) * XS + 16 * kt + 2 * q;
    a[0] = *reinterpret_cast<const uint32_t*>(p);
    a[1] = *reinterpret_cast<const uint32_t*>(p + 8 * XS);
    a[2] = *reinterpret_cast<const uint32_t*>(p + 8);
    a[3] = *reinterpret_cast<const uint32_t*>(p + 8 * XS + 8);
}

// A fragment of the TRANSPOSE of a [k][m] row-major bf16 tile: A(m, k) = T[k][m]
__device__ __forceinline__ void afrag_t(const __nv_bfloat16* T, int mt, int kt, int g, int q, uint32_t a[4]) {
    int m0 = 16 * mt + g, k0 = 16 * kt + 2 * q;
    a[0] = pack_bf16_raw(T[k0 * XS + m0], T[(k0 + 1) * XS + m0]);
    a[1] = pack_bf16_raw(T[k0 * XS + m0 + 8], T[(k0 + 1) * XS + m0 + 8]);
    a[2] = pack_bf16_raw(T[(k0 + 8) * XS + m0], T[(k0 + 9) * XS + m0]);
    a[3] = pack_bf16_raw(T[(k0 + 8) * XS + m0 + 8], T[(k0 + 9) * XS + m0 + 8]);
}

// B fragment of a [k][n] row-major bf16 tile: B(k, n) = T[k][n]
__device__ __forceinline__ void bfrag_kn(const __nv_bfloat16* T, int nt, int kt, int g, int q, uint32_t b[2]) {
    int n = 8 * nt + g, k0 = 16 * kt + 2 * q;
    b[0] = pack_bf16_raw(T[k0 * XS + n], T[(k0 + 1) * XS + n]);
    b[1] = pack_bf16_raw(T[(k0 + 8) * XS + n], T[(k0 + 9) * XS + n]);
}

// Forward of one warp's 32 rows.  X: the warp's [32][XS] bf16 input tile.
// z1/z2: pre-activations in accumulator layout [mt][nt][4]; h1a: layer-2 A
// fragments (GELU(z1) as bf16); logit for rows (16 mt + g) and (16 mt + g + 8)
// is returned in lg[mt][0..1] on every lane of the quad.
struct MlpFwd {
    float z1[2][4][4], z2[2][4][4];
    uint32_t h1a[2][2][4];
    float lg[2][2];
};

__device__ __forceinline__ void mlp_forward(const MlpSmem& m, const __nv_bfloat16* X, MlpFwd& f) {
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
        uint32_t a[2][4];
        afrag(X, mt, 0, g, q, a[0]);
        afrag(X, mt, 1, g, q, a[1]);
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            float* d = f.z1[mt][nt];
            float bl = m.b1[8 * nt + 2 * q], bh = m.b1[8 * nt + 2 * q + 1];
            d[0] = bl; d[1] = bh; d[2] = bl; d[3] = bh;
#pragma unroll
            for (int kt = 0; kt < 2; kt++) {
                uint32_t b[2];
                bfrag(m.W1, nt, kt, g, q, b);
                mma16816(d, a[kt], b);
            }
        }
        // accumulator tiles (2t, 2t+1) are the A fragment of k-tile t of layer 2
#pragma unroll
        for (int t = 0; t < 2; t++) {
            const float* c0 = f.z1[mt][2 * t];
            const float* c1 = f.z1[mt][2 * t + 1];
            f.h1a[mt][t][0] = pack_bf16(gelu(c0[0]), gelu(c0[1]));
            f.h1a[mt][t][1] = pack_bf16(gelu(c0[2]), gelu(c0[3]));
            f.h1a[mt][t][2] = pack_bf16(gelu(c1[0]), gelu(c1[1]));
            f.h1a[mt][t][3] = pack_bf16(gelu(c1[2]), gelu(c1[3]));
        }
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            float* d = f.z2[mt][nt];
            float bl = m.b2[8 * nt + 2 * q], bh = m.b2[8 * nt + 2 * q + 1];
            d[0] = bl; d[1] = bh; d[2] = bl; d[3] = bh;
#pragma unroll
            for (int kt = 0; kt < 2; kt++) {
                uint32_t b[2];
                bfrag(m.W2, nt, kt, g, q, b);
                mma16816(d, f.h1a[mt][kt], b);
            }
        }
        float s0 = 0.f, s1 = 0.f;
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            float wl = m.w3[8 * nt + 2 * q], wh = m.w3[8 * nt + 2 * q + 1];
            s0 += gelu(f.z2[mt][nt][0]) * wl + gelu(f.z2[mt][nt][1]) * wh;
            s1 += gelu(f.z2[mt][nt][2]) * wl + gelu(f.z2[mt][nt][3]) * wh;
        }
        s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
        s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
        s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
        s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
        f.lg[mt][0] = s0 + m.b3;
        f.lg[mt][1] = s1 + m.b3;
    }
}

// Inference-only forward for the per-step flags: GELU on packed BF16 pairs
// (tanh.approx.bf16x2 and bf16x2 FMAs: half the special-function and FMA
// instructions of the FP32 GELU).  The layer-1 activations feed layer 2 as
// BF16 either way; the layer-2 activations are widened to FP32 for the output
// dot product.  Training and ns_sensor_predict use the FP32 GELU above.
__device__ __forceinline__ __nv_bfloat162 tanh_bf16x2(__nv_bfloat162 x) {
    uint32_t xi = *reinterpret_cast<uint32_t*>(&x), yi;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(yi) : "r"(xi));
    return *reinterpret_cast<__nv_bfloat162*>(&yi);
}
__device__ __forceinline__ __nv_bfloat162 gelu_bf16x2(float a, float b) {
    const __nv_bfloat162 x = __floats2bfloat162_rn(a, b);
    const __nv_bfloat162 c0 = __float2bfloat162_rn(0.7978845608028654f);
    const __nv_bfloat162 c1 = __float2bfloat162_rn(0.7978845608028654f * 0.044715f);
    const __nv_bfloat162 half = __float2bfloat162_rn(0.5f);
    const __nv_bfloat162 u = __hmul2(x, __hfma2(__hmul2(x, x), c1, c0));  // k0 (x + k1 x^3)
    const __nv_bfloat162 h = __hmul2(half, x);
    return __hfma2(h, tanh_bf16x2(u), h);
}

// ---------------------------------------------------------------------------
// features

template <typename T>
__device__ __forceinline__ void face_features(const T rho[6], const T p[6], const T un[6], float gamma,
                                              float feat[SF]) {
    float mr = 0.f, mp = 0.f, mu = 0.f;
#pragma unroll
    for (int s = 0; s < 6; s++) { mr += float(rho[s]); mp += float(p[s]); mu += float(un[s]); }
    mr *= (1.f / 6.f); mp *= (1.f / 6.f); mu *= (1.f / 6.f);
    float cs = sqrtf(fmaxf(gamma * mp / fmaxf(mr, 1e-30f), 0.f));
    const float* none = nullptr;
    (void)none;
    float scale[3] = {1e-3f * fabsf(mr), 1e-3f * fabsf(mp), 1e-3f * cs + 1e-30f};
    float mean[3] = {mr, mp, mu};
#pragma unroll
    for (int v = 0; v < 3; v++) {
        float d[6], mx = 0.f;
#pragma unroll
        for (int s = 0; s < 6; s++) {
            float x = v == 0 ? float(rho[s]) : (v == 1 ? float(p[s]) : float(un[s]));
            d[s] = x - mean[v];
            mx = fmaxf(mx, fabsf(d[s]));
        }
        float inv = __fdividef(1.f, mx + scale[v] + 1e-30f);
#pragma unroll
        for (int s = 0; s < 6; s++) feat[6 * v + s] = d[s] * inv;
    }
    float b0, b1, b2;
    weno_betas<float>(float(rho[0]), float(rho[1]), float(rho[2]), float(rho[3]), float(rho[4]), b0, b1, b2);
    float den = b0 + b1 + b2 + (1e-3f * mr) * (1e-3f * mr) + 1e-30f;
    float iden = __fdividef(1.f, den);
    feat[18] = b0 * iden;
    feat[19] = b1 * iden;
    feat[20] = b2 * iden;
}

// rho, p and u_n of the 6-cell stencil of a face
template <int DIR, typename T>
__device__ __forceinline__ void face_prims(const double* __restrict__ W, const Box& b, long long o0,
                                           long long step, T rho[6], T p[6], T un[6]) {
#pragma unroll
    for (int s = 0; s < 6; s++) {
        long long o = o0 + s * step;
        rho[s] = T(W[o]);
        p[s] = T(W[b.fstride + o]);
        un[s] = T(W[(2 + DIR) * b.fstride + o]);
    }
}

// ---------------------------------------------------------------------------
// harvest: features + label of every face along DIR (FP64 fluxes of the
// context's semantics: PHYS selects the physical form's fluxes)

template <int DIR, bool BORGES, bool PHYS>
__global__ void __launch_bounds__(128) k_sensor_harvest(const double* __restrict__ W,
                                                        const double* __restrict__ U, Box b, Consts c,
                                                        FaceBox fb, long long base, double thr,
                                                        float* __restrict__ feat,
                                                        float* __restrict__ label) {
    int kk = blockIdx.x * 32 + threadIdx.x;
    int bb = blockIdx.y * 4 + threadIdx.y;
    int aa = blockIdx.z;
    if (kk >= fb.n2 || bb >= fb.n1) return;
    long long step;
    long long o0 = face_origin<DIR>(b, aa, bb, kk, step);
    double fL[5][5], fR[5][5], wa[5], fc[5], fx[5];
    face_stencil<DIR, true, PHYS, double>(W, U, b, c, o0, step, fL, fR, wa);
    face_comp<double, BORGES>(fL, fR, fc);
    face_char<DIR, PHYS, double, BORGES>(fL, fR, wa, c.gamma, c.inv_gm1, fx);
    double dn = 0, nn = 0;
#pragma unroll
    for (int q = 0; q < 5; q++) {
        dn += (fx[q] - fc[q]) * (fx[q] - fc[q]);
        nn += fx[q] * fx[q];
    }
    long long idx = base + fb.at(aa, bb, kk);
    label[idx] = (sqrt(dn) > thr * (sqrt(nn) + 1e-12)) ? 1.f : 0.f;
    float rho[6], p[6], un[6], f[SF];
    face_prims<DIR, float>(W, b, o0, step, rho, p, un);
    face_features<float>(rho, p, un, float(c.gamma), f);
#pragma unroll
    for (int e = 0; e < SF; e++) feat[idx * SF + e] = f[e];
}

// ---------------------------------------------------------------------------
// training: fused forward + backward of 128 samples per block (4 warps x 32),
// BCE-with-logits loss with positive-class weight, gradients summed in shared
// memory then added to the global FP32 gradient.

struct TrainSmem {
    MlpSmem m;
    __nv_bfloat16 X[4][32 * XS];   // per warp: inputs
    __nv_bfloat16 H[4][32 * XS];   // per warp: GELU(z1) (then reused)
    __nv_bfloat16 D[4][32 * XS];   // per warp: dZ2, then dZ1
    float grad[SP];
    float loss;
};

__device__ __forceinline__ unsigned long long perm_index(unsigned long long i, unsigned long long n,
                                                         unsigned long long a, unsigned long long c) {
    return (a * i + c) % n;  // a coprime with n: a bijection of [0, n)
}

__global__ void __launch_bounds__(128) k_mlp_train(const float* __restrict__ feat,
                                                   const float* __restrict__ label, long long n,
                                                   long long start, int count, unsigned long long pa,
                                                   unsigned long long pc, float pos_weight,
                                                   float inv_batch, const float* __restrict__ w,
                                                   float* __restrict__ grad, float* __restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, q = lane & 3;
    mlp_load(S.m, w, true);
    for (int e = tid; e < SP; e += blockDim.x) S.grad[e] = 0.f;
    if (tid == 0) S.loss = 0.f;
    // inputs of this warp's 32 samples (rows beyond count are zero with zero weight)
    const int row0 = blockIdx.x * 128 + warp * 32;
    __nv_bfloat16* X = S.X[warp];
    float yv = 0.f, valid = 0.f;
    {
        int r = row0 + lane;
        bool ok = r < count;
        long long src = ok ? (long long)perm_index((unsigned long long)(start + r), (unsigned long long)n, pa, pc) : 0;
        for (int e = 0; e < XS; e++) X[lane * XS + e] = __float2bfloat16(ok && e < SF ? feat[src * SF + e] : 0.f);
        yv = ok ? label[src] : 0.f;
        valid = ok ? 1.f : 0.f;
    }
    __syncthreads();
    MlpFwd f;
    mlp_forward(S.m, X, f);
    // per-row dL/dz for rows (16mt+g) and (16mt+g+8): fetch label/valid from the owning lanes
    float dz[2][2];
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
            int r = 16 * mt + g + 8 * h;
            float y = __shfl_sync(0xffffffffu, yv, r);
            float ok = __shfl_sync(0xffffffffu, valid, r);
            float z = f.lg[mt][h];
            float sg = 1.f / (1.f + __expf(-z));
            // loss = pw y softplus(-z) + (1-y) softplus(z); dloss/dz = sg (pw y + 1 - y) - pw y
            float sp_pos = fmaxf(-z, 0.f) + log1pf(__expf(-fabsf(z)));
            float sp_neg = fmaxf(z, 0.f) + log1pf(__expf(-fabsf(z)));
            float l = pos_weight * y * sp_pos + (1.f - y) * sp_neg;
            dz[mt][h] = ok * inv_batch * (sg * (pos_weight * y + 1.f - y) - pos_weight * y);
            if (q == 0 && ok > 0.f) atomicAdd(&S.loss, l * inv_batch);
        }
    // layer 3 and dZ2
    float dz2[2][4][4];
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                int col = 8 * nt + 2 * q + (e & 1);
                float d = dz[mt][e >> 1];
                float z2 = f.z2[mt][nt][e];
                // dw3 += dz * h2, db2 += dz2
                atomicAdd(&S.grad[OFF_W3 + col], d * gelu(z2));
                dz2[mt][nt][e] = d * S.m.w3[col] * gelu_grad(z2);
                atomicAdd(&S.grad[OFF_B2 + col], dz2[mt][nt][e]);
            }
    if (q == 0)
#pragma unroll
        for (int mt = 0; mt < 2; mt++) atomicAdd(&S.grad[OFF_B3], dz[mt][0] + dz[mt][1]);
    // stage H1 = GELU(z1) and dZ2 as [sample][unit] bf16 tiles
    __nv_bfloat16* H = S.H[warp];
    __nv_bfloat16* D = S.D[warp];
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                int r = 16 * mt + g + 8 * (e >> 1), col = 8 * nt + 2 * q + (e & 1);
                H[r * XS + col] = __float2bfloat16(gelu(f.z1[mt][nt][e]));
                D[r * XS + col] = __float2bfloat16(dz2[mt][nt][e]);
            }
    __syncwarp();
    // dW2[out][in] += sum_s dZ2[s][out] H1[s][in]: M = out, N = in, K = samples
#pragma unroll
    for (int mo = 0; mo < 2; mo++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int ks = 0; ks < 2; ks++) {
                uint32_t a[4], bb[2];
                afrag_t(D, mo, ks, g, q, a);
                bfrag_kn(H, ni, ks, g, q, bb);
                mma16816(acc, a, bb);
            }
#pragma unroll
            for (int e = 0; e < 4; e++) {
                int o = 16 * mo + g + 8 * (e >> 1), i = 8 * ni + 2 * q + (e & 1);
                atomicAdd(&S.grad[OFF_W2 + o * 32 + i], acc[e]);
            }
        }
    // dH1 = dZ2 W2 (M = samples, N = in, K = out): A = dZ2 from the accumulator layout
    float dz1[2][4][4];
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
        uint32_t a[2][4];
#pragma unroll
        for (int t = 0; t < 2; t++) {
            a[t][0] = pack_bf16(dz2[mt][2 * t][0], dz2[mt][2 * t][1]);
            a[t][1] = pack_bf16(dz2[mt][2 * t][2], dz2[mt][2 * t][3]);
            a[t][2] = pack_bf16(dz2[mt][2 * t + 1][0], dz2[mt][2 * t + 1][1]);
            a[t][3] = pack_bf16(dz2[mt][2 * t + 1][2], dz2[mt][2 * t + 1][3]);
        }
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kt = 0; kt < 2; kt++) {
                uint32_t bb[2];
                bfrag(S.m.W2T, nt, kt, g, q, bb);  // B(k = out, n = in) = W2[out][in] = W2T[in][out]
                mma16816(acc, a[kt], bb);
            }
#pragma unroll
            for (int e = 0; e < 4; e++) {
                int col = 8 * nt + 2 * q + (e & 1);
                dz1[mt][nt][e] = acc[e] * gelu_grad(f.z1[mt][nt][e]);
                atomicAdd(&S.grad[OFF_B1 + col], dz1[mt][nt][e]);
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                int r = 16 * mt + g + 8 * (e >> 1), col = 8 * nt + 2 * q + (e & 1);
                D[r * XS + col] = __float2bfloat16(dz1[mt][nt][e]);
            }
    __syncwarp();
    // dW1[out][in] += sum_s dZ1[s][out] X[s][in]
#pragma unroll
    for (int mo = 0; mo < 2; mo++)
#pragma unroll
        for (int ni = 0; ni < 3; ni++) {  // in-columns 0..23 cover the 21 features
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int ks = 0; ks < 2; ks++) {
                uint32_t a[4], bb[2];
                afrag_t(D, mo, ks, g, q, a);
                bfrag_kn(X, ni, ks, g, q, bb);
                mma16816(acc, a, bb);
            }
#pragma unroll
            for (int e = 0; e < 4; e++) {
                int o = 16 * mo + g + 8 * (e >> 1), i = 8 * ni + 2 * q + (e & 1);
                if (i < SF) atomicAdd(&S.grad[OFF_W1 + o * 32 + i], acc[e]);
            }
        }
    __syncthreads();
    for (int e = tid; e < SP; e += blockDim.x)
        if (S.grad[e] != 0.f) atomicAdd(&grad[e], S.grad[e]);
    if (tid == 0) atomicAdd(loss, S.loss);
}

// Adam (Kingma & Ba 2015) on the FP32 master weights; clears the gradient
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       float* __restrict__ grad, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    for (int e = threadIdx.x + blockIdx.x * blockDim.x; e < SP; e += blockDim.x * gridDim.x) {
        float gr = grad[e];
        grad[e] = 0.f;
        bool unused = (e < OFF_B1) && ((e % 32) >= SF);  // padded input columns of W1 stay zero
        if (unused) continue;
        float mm = b1 * m[e] + (1.f - b1) * gr;
        float vv = b2 * v[e] + (1.f - b2) * gr * gr;
        m[e] = mm;
        v[e] = vv;
        w[e] -= lr * (mm * c1) / (sqrtf(vv * c2) + eps);
    }
}

// logits of n samples (4 warps x 32 samples per block)
__global__ void __launch_bounds__(128) k_mlp_predict(const float* __restrict__ feat, long long n,
                                                     const float* __restrict__ w,
                                                     float* __restrict__ logit) {
    __shared__ __align__(16) MlpSmem m;
    __shared__ __align__(16) __nv_bfloat16 Xs[4][32 * XS];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, q = lane & 3;
    mlp_load(m, w, false);
    long long r = (long long)blockIdx.x * 128 + warp * 32 + lane;
    __nv_bfloat16* X = Xs[warp];
    for (int e = 0; e < XS; e++) X[lane * XS + e] = __float2bfloat16(r < n && e < SF ? feat[r * SF + e] : 0.f);
    __syncthreads();
    MlpFwd f;
    mlp_forward(m, X, f);
    if (q == 0) {
        long long base = (long long)blockIdx.x * 128 + warp * 32;
#pragma unroll
        for (int mt = 0; mt < 2; mt++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                long long rr = base + 16 * mt + g + 8 * h;
                if (rr < n) logit[rr] = f.lg[mt][h];
            }
    }
}

// ---------------------------------------------------------------------------
// gated FP32 face flux: component-wise everywhere, MLP on the tensor cores,
// characteristic-wise recomputed on the flagged faces of the block (compacted
// into a shared-memory list so the recompute runs without divergence).

template <int DIR, bool BORGES, bool PHYS>
__global__ void __launch_bounds__(128) k_face_gated(const double* __restrict__ W,
                                                    const double* __restrict__ U, Box b, Consts c,
                                                    float* __restrict__ F, FaceBox fb,
                                                    const float* __restrict__ w, float logit_thr,
                                                    unsigned long long* __restrict__ flagged) {
    __shared__ __align__(16) MlpSmem m;
    __shared__ __align__(16) __nv_bfloat16 Xs[4][32 * XS];
    __shared__ int list[128];
    __shared__ int nlist;
    const int tid = threadIdx.x + 32 * threadIdx.y, warp = threadIdx.y, lane = threadIdx.x;
    const int g = lane >> 2, q = lane & 3;
    mlp_load(m, w, false);
    if (tid == 0) nlist = 0;
    int kk = blockIdx.x * 32 + threadIdx.x;
    int bb = blockIdx.y * 4 + threadIdx.y;
    int aa = blockIdx.z;
    const bool live = kk < fb.n2 && bb < fb.n1;
    long long step = 0, o0 = 0;
    float feat[SF];
    if (live) {
        o0 = face_origin<DIR>(b, aa, bb, kk, step);
        float fL[5][5], fR[5][5], wa[5], out[5];
        face_stencil<DIR, false, PHYS, float>(W, U, b, c, o0, step, fL, fR, wa);
        face_comp<float, BORGES>(fL, fR, out);
        long long fo = fb.at(aa, bb, kk);
#pragma unroll
        for (int qq = 0; qq < 5; qq++) F[qq * fb.fstride + fo] = out[qq];
        float rho[6], p[6], un[6];
        face_prims<DIR, float>(W, b, o0, step, rho, p, un);
        face_features<float>(rho, p, un, float(c.gamma), feat);
    } else {
#pragma unroll
        for (int e = 0; e < SF; e++) feat[e] = 0.f;
    }
    __nv_bfloat16* X = Xs[warp];
#pragma unroll
    for (int e = 0; e < XS; e++) X[lane * XS + e] = __float2bfloat16(e < SF ? feat[e] : 0.f);
    __syncthreads();
    MlpFwd f;
    mlp_forward(m, X, f);
    // the logit of this lane's face (row = lane) sits with lane 4*(row%8) of tile row/16, half (row%16)/8
    float lg = 0.f;
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
            float v = __shfl_sync(0xffffffffu, f.lg[mt][h], 4 * (lane & 7));
            if ((lane >> 4) == mt && ((lane >> 3) & 1) == h) lg = v;
        }
    (void)g; (void)q;
    bool fire = live && lg > logit_thr;
    unsigned mask = __ballot_sync(0xffffffffu, fire);
    int nfire = __popc(mask);
    int slot = 0;
    if (lane == 0 && nfire) slot = atomicAdd(&nlist, nfire);
    slot = __shfl_sync(0xffffffffu, slot, 0);
    if (fire) list[slot + __popc(mask & ((1u << lane) - 1u))] = (threadIdx.y << 5) | threadIdx.x;
    __syncthreads();
    const int n = nlist;
    if (tid == 0 && n) atomicAdd(flagged, (unsigned long long)n);
    for (int e = tid; e < n; e += 128) {
        int t = list[e];
        int k2 = blockIdx.x * 32 + (t & 31), b2 = blockIdx.y * 4 + (t >> 5);
        long long st2;
        long long p0 = face_origin<DIR>(b, aa, b2, k2, st2);
        float fL[5][5], fR[5][5], wa[5], out[5];
        face_stencil<DIR, true, PHYS, float>(W, U, b, c, p0, st2, fL, fR, wa);
        face_char<DIR, PHYS, float, BORGES>(fL, fR, wa, float(c.gamma), float(c.inv_gm1), out);
        long long fo = fb.at(aa, b2, k2);
#pragma unroll
        for (int qq = 0; qq < 5; qq++) F[qq * fb.fstride + fo] = out[qq];
    }
}

// ---------------------------------------------------------------------------
// per-step flags for the fused stage kernel: the MLP on every face along DIR of
// the step's start state U0 (W = prim(U0) at boundary-folded cells, the
// stage kernel's own halo rule), one byte per face (1 = characteristic-wise)

// rho, p, u, v, w of every interior cell in FP32 (what the flags' features read),
// SoA planes of nx*ny*nz floats, from the step's start state U0
__global__ void __launch_bounds__(128) k_sensor_prims(const double* __restrict__ U0, Box b, Consts c,
                                                      float* __restrict__ prim) {
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 4 + threadIdx.y, i = blockIdx.z;
    if (k >= b.nz || j >= b.ny) return;
    const long long o = b.at(i + NG, j + NG, k + NG);
    const long long n = (long long)b.nx * b.ny * b.nz, e = ((long long)i * b.ny + j) * b.nz + k;
    float u[5];
#pragma unroll
    for (int q = 0; q < 5; q++) u[q] = float(U0[q * b.fstride + o]);
    const float ir = __fdividef(1.f, u[0]);
    prim[e] = u[0];
    prim[n + e] = float(c.gm1) * (u[1] - 0.5f * ir * (u[2] * u[2] + u[3] * u[3] + u[4] * u[4]));
    prim[2 * n + e] = u[2] * ir;
    prim[3 * n + e] = u[3] * ir;
    prim[4 * n + e] = u[4] * ir;
}

// Flags of every face along DIR on the 5th-generation tensor cores; a flagged
// face also goes into the compacted list of its axis (FaceBox index) and marks
// the interior cells on either side as touched, for the correction passes of
// ns_gate.cu.  A CTA of 128 threads takes
// 128 faces per tile; their BF16 features (K = 32, the 21 features and zeros)
// and the network's weight tiles sit in shared memory in the K-major layout, one
// thread issues two K = 16 tcgen05.mma per layer (M = 128 faces, N = 32 hidden
// units, FP32 accumulators in 32 TMEM columns) and commits them to an
// mbarrier, and every thread reads its face's 32 pre-activations back with
// tcgen05.ld for the bias, the GELU and the next layer's operand.  A wait that
// runs out of polls sets *err and ends the kernel after freeing its TMEM.
constexpr uint32_t kMmaPolls = 1u << 24;

template <int DIR>
__global__ void __launch_bounds__(128) k_sensor_mask_tc(const float* __restrict__ prim, Box b, Consts c,
                                                        FaceBox fb, const float* __restrict__ w,
                                                        float logit_thr, unsigned char* __restrict__ mask,
                                                        unsigned long long* __restrict__ flagged,
                                                        unsigned* __restrict__ list, unsigned* __restrict__ count,
                                                        unsigned char* __restrict__ touched, int* __restrict__ err) {
    __shared__ __align__(128) unsigned char A1[128 * 32 * 2];
    __shared__ __align__(128) unsigned char A2[128 * 32 * 2];
    __shared__ __align__(128) unsigned char B1[32 * 32 * 2];
    __shared__ __align__(128) unsigned char B2[32 * 32 * 2];
    __shared__ float vb1[SH], vb2[SH], vw3[SH];
    __shared__ float vb3;
    __shared__ __align__(8) unsigned long long bar;
    __shared__ uint32_t tslot;
    const int warp = threadIdx.y, lane = threadIdx.x, tid = warp * 32 + lane;
    // weight tiles [n][k] in the K-major layout (W1's columns past the 21 features are zero)
    for (int e = tid; e < SH * 32; e += 128) {
        const int n = e >> 5, k = e & 31;
        *reinterpret_cast<__nv_bfloat16*>(B1 + tc::kmajor_offset<32>(n, k)) =
            __float2bfloat16(k < SF ? w[OFF_W1 + n * 32 + k] : 0.f);
        *reinterpret_cast<__nv_bfloat16*>(B2 + tc::kmajor_offset<32>(n, k)) = __float2bfloat16(w[OFF_W2 + n * 32 + k]);
    }
    if (tid < SH) {
        vb1[tid] = w[OFF_B1 + tid];
        vb2[tid] = w[OFF_B2 + tid];
        vw3[tid] = w[OFF_W3 + tid];
    }
    if (tid == 0) vb3 = w[OFF_B3];
    const uint32_t bar_a = tc::smem_u32(&bar);
    if (tid == 0) tc::mbar_init(bar_a, 1);
    if (warp == 0) tc::tmem_alloc(tc::smem_u32(&tslot), 32);
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tslot;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's 32 lanes
    constexpr uint32_t idesc = tc::idesc_bf16_f32<128, 32>();
    // K halves: A tiles (128 rows) 2 x 2048 B apart, B tiles (32 rows) 2 x 512 B apart
    const uint64_t dA1[2] = {tc::kmajor_desc(tc::smem_u32(A1), 2048, 128), tc::kmajor_desc(tc::smem_u32(A1) + 4096, 2048, 128)};
    const uint64_t dA2[2] = {tc::kmajor_desc(tc::smem_u32(A2), 2048, 128), tc::kmajor_desc(tc::smem_u32(A2) + 4096, 2048, 128)};
    const uint64_t dB1[2] = {tc::kmajor_desc(tc::smem_u32(B1), 512, 128), tc::kmajor_desc(tc::smem_u32(B1) + 1024, 512, 128)};
    const uint64_t dB2[2] = {tc::kmajor_desc(tc::smem_u32(B2), 512, 128), tc::kmajor_desc(tc::smem_u32(B2) + 1024, 512, 128)};
    const float gamma = float(c.gamma);
    const unsigned t2 = (fb.n2 + 31) / 32, t1 = (fb.n1 + 3) / 4, t12 = t2 * t1;
    const unsigned tiles = t12 * (unsigned)fb.n0;
    const long long n = (long long)b.nx * b.ny * b.nz;
    uint32_t phase = 0;
    bool ok = true;
    unsigned long long nfire = 0;
    for (unsigned t = blockIdx.x; t < tiles; t += gridDim.x) {
        const unsigned aa_ = t / t12, r = t - aa_ * t12, b1 = r / t2;
        const int kk = (int)(r - b1 * t2) * 32 + lane;
        const int bb = (int)b1 * 4 + warp;
        const int aa = (int)aa_;
        const bool live = kk < fb.n2 && bb < fb.n1;
        float feat[32];
#pragma unroll
        for (int e = 0; e < 32; e++) feat[e] = 0.f;
        if (live) {
            float rho[6], p[6], un[6];
#pragma unroll
            for (int s = 0; s < 6; s++) {
                int i = aa, j = bb, k = kk;
                if (DIR == 0) i = fold(aa - 3 + s, b.nx, c.periodic[0]);
                if (DIR == 1) j = fold(bb - 3 + s, b.ny, c.periodic[1]);
                if (DIR == 2) k = fold(kk - 3 + s, b.nz, c.periodic[2]);
                const long long e = ((long long)i * b.ny + j) * b.nz + k;
                rho[s] = prim[e];
                p[s] = prim[n + e];
                un[s] = prim[(2 + DIR) * n + e];
            }
            face_features<float>(rho, p, un, gamma, feat);
        }
        // this face is row tid of the A tile: four 16-byte chunks of 8 features
#pragma unroll
        for (int kb = 0; kb < 4; kb++) {
            uint32_t q[4];
#pragma unroll
            for (int h = 0; h < 4; h++) q[h] = pack_bf16(feat[8 * kb + 2 * h], feat[8 * kb + 2 * h + 1]);
            *reinterpret_cast<uint4*>(A1 + tc::kmajor_offset<128>(tid, 8 * kb)) = make_uint4(q[0], q[1], q[2], q[3]);
        }
        tc::fence_smem_to_async();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) {
            tc::mma_bf16(tmem, dA1[0], dB1[0], idesc, false);
            tc::mma_bf16(tmem, dA1[1], dB1[1], idesc, true);
            tc::commit_to(bar_a);
        }
        ok = tc::mbar_wait(bar_a, phase, kMmaPolls) && ok;
        phase ^= 1;
        tc::fence_after_sync();
        float d[32];
        tc::tmem_ld32(trow, d);
        // layer 1: GELU(z + b1) as the second layer's BF16 operand, row tid
#pragma unroll
        for (int kb = 0; kb < 4; kb++) {
            uint32_t q[4];
#pragma unroll
            for (int h = 0; h < 4; h++) {
                const int e = 8 * kb + 2 * h;
                __nv_bfloat162 v = gelu_bf16x2(d[e] + vb1[e], d[e + 1] + vb1[e + 1]);
                q[h] = *reinterpret_cast<uint32_t*>(&v);
            }
            *reinterpret_cast<uint4*>(A2 + tc::kmajor_offset<128>(tid, 8 * kb)) = make_uint4(q[0], q[1], q[2], q[3]);
        }
        tc::fence_smem_to_async();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) {
            tc::mma_bf16(tmem, dA2[0], dB2[0], idesc, false);
            tc::mma_bf16(tmem, dA2[1], dB2[1], idesc, true);
            tc::commit_to(bar_a);
        }
        ok = tc::mbar_wait(bar_a, phase, kMmaPolls) && ok;
        phase ^= 1;
        tc::fence_after_sync();
        tc::tmem_ld32(trow, d);
        float lg = vb3;
#pragma unroll
        for (int e = 0; e < 32; e += 2) {
            const float2 g = __bfloat1622float2(gelu_bf16x2(d[e] + vb2[e], d[e + 1] + vb2[e + 1]));
            lg = fmaf(g.x, vw3[e], fmaf(g.y, vw3[e + 1], lg));
        }
        const bool fire = live && lg > logit_thr;
        const long long fi = live ? fb.at(aa, bb, kk) : 0;
        if (live) mask[fi] = fire ? 1 : 0;
        const unsigned m = __ballot_sync(0xffffffffu, fire);
        nfire += __popc(m);
        if (m) {
            unsigned base = 0;
            if (lane == 0) base = atomicAdd(count, (unsigned)__popc(m));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (fire) {
                list[base + __popc(m & ((1u << lane) - 1u))] = (unsigned)fi;
                const int a = DIR == 0 ? aa : (DIR == 1 ? bb : kk), na = DIR == 0 ? b.nx : (DIR == 1 ? b.ny : b.nz);
                const long long cell = ((long long)aa * b.ny + bb) * b.nz + kk;
                const long long step = DIR == 0 ? (long long)b.ny * b.nz : (DIR == 1 ? (long long)b.nz : 1LL);
                if (a - 1 >= 0) touched[cell - step] = 1;
                if (a < na) touched[cell] = 1;
            }
        }
        tc::fence_before_sync();  // this tile's TMEM reads precede the next tile's MMA
        if (!__syncthreads_and(ok)) break;
    }
    if (!ok && tid == 0) atomicExch(err, 1);
    if (lane == 0 && nfire) atomicAdd(flagged, nfire);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_free(tmem, 32);
}

// compacted list of the touched cells (interior order), the cells a correction pass updates
__global__ void __launch_bounds__(128) k_sensor_touched_list(const unsigned char* __restrict__ touched, long long n,
                                                             unsigned* __restrict__ list, unsigned* __restrict__ count) {
    const long long e = (long long)blockIdx.x * 128 + threadIdx.x;
    const bool t = e < n && touched[e] != 0;
    const unsigned m = __ballot_sync(0xffffffffu, t);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(count, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (t) list[base + __popc(m & ((1u << lane) - 1u))] = (unsigned)e;
}

// ---------------------------------------------------------------------------
// context-side state

struct SensorState {
    float* w = nullptr;                    // FP32 parameters on the device
    unsigned long long* flagged = nullptr;  // faces flagged since creation
    unsigned char* mask[3] = {nullptr, nullptr, nullptr};  // per-step flags, one byte per face
    unsigned* list[3] = {nullptr, nullptr, nullptr};       // flagged faces per axis (compacted)
    unsigned* counts = nullptr;            // [0..2] flagged faces per axis, [3] touched cells
    unsigned char* touched = nullptr;      // cells next to a flagged face, one byte per interior cell
    unsigned* cells = nullptr;             // the touched cells (compacted)
    long long ncells = 0;
    int* err = nullptr;                    // set by a tensor-core wait that ran out of polls
    float* prim = nullptr;                  // the step's rho, p, u, v, w (FP32 planes) for the flags
    unsigned long long faces = 0;           // faces evaluated since creation (host count)
    int sms = 148;                          // multiprocessors of the context's device
    bool has_weights = false;
};

ns_status sensor_create(SensorState** out, const Box& b, const FaceBox* fb, cudaStream_t s) {
    *out = nullptr;
    SensorState* st = new (std::nothrow) SensorState();
    if (!st) return NS_ERR_OOM;
    bool ok = cudaMalloc(&st->w, SP * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&st->flagged, sizeof(unsigned long long)) == cudaSuccess;
    for (int d = 0; d < 3 && ok; d++) ok = cudaMalloc(&st->mask[d], (size_t)fb[d].fstride) == cudaSuccess;
    for (int d = 0; d < 3 && ok; d++)
        ok = cudaMalloc(&st->list[d], (size_t)fb[d].fstride * sizeof(unsigned)) == cudaSuccess;
    st->ncells = (long long)b.nx * b.ny * b.nz;
    ok = ok && cudaMalloc(&st->err, sizeof(int)) == cudaSuccess &&
         cudaMalloc(&st->counts, 4 * sizeof(unsigned)) == cudaSuccess &&
         cudaMalloc(&st->touched, (size_t)st->ncells) == cudaSuccess &&
         cudaMalloc(&st->cells, (size_t)st->ncells * sizeof(unsigned)) == cudaSuccess;
    ok = ok && cudaMalloc(&st->prim, (size_t)5 * b.nx * b.ny * b.nz * sizeof(float)) == cudaSuccess;
    int dev = 0;
    if (ok && cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&st->sms, cudaDevAttrMultiProcessorCount, dev);
    if (!ok) {
        sensor_destroy(st);
        cudaGetLastError();
        return NS_ERR_OOM;
    }
    cudaMemsetAsync(st->w, 0, SP * sizeof(float), s);
    cudaMemsetAsync(st->flagged, 0, sizeof(unsigned long long), s);
    cudaMemsetAsync(st->counts, 0, 4 * sizeof(unsigned), s);
    cudaMemsetAsync(st->err, 0, sizeof(int), s);
    *out = st;
    return NS_OK;
}

void sensor_destroy(SensorState* st) {
    if (!st) return;
    cudaFree(st->w);
    cudaFree(st->flagged);
    for (int d = 0; d < 3; d++) cudaFree(st->mask[d]);
    for (int d = 0; d < 3; d++) cudaFree(st->list[d]);
    cudaFree(st->counts);
    cudaFree(st->err);
    cudaFree(st->touched);
    cudaFree(st->cells);
    cudaFree(st->prim);
    delete st;
}

ns_status sensor_set_weights(SensorState* st, const float* w, cudaStream_t s) {
    if (cudaMemcpyAsync(st->w, w, SP * sizeof(float), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return NS_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return NS_ERR_CUDA;
    st->has_weights = true;
    return NS_OK;
}

ns_status sensor_face_flux(SensorState* st, int dir, const double* W, const double* U, const Box& b,
                           const Consts& c, double threshold, bool borges, bool phys, void* F,
                           const FaceBox& fb, cudaStream_t s, long long* launches) {
    const float thr = (float)std::log(threshold / (1.0 - threshold));
    dim3 grid((fb.n2 + 31) / 32, (fb.n1 + 3) / 4, fb.n0), blk(32, 4);
#define NS_GATED1(D, B, PH) \
    k_face_gated<D, B, PH><<<grid, blk, 0, s>>>(W, U, b, c, (float*)F, fb, st->w, thr, st->flagged)
#define NS_GATED(D)                                               \
    do {                                                          \
        if (phys) {                                               \
            if (borges) NS_GATED1(D, true, true);                 \
            else NS_GATED1(D, false, true);                       \
        } else {                                                  \
            if (borges) NS_GATED1(D, true, false);                \
            else NS_GATED1(D, false, false);                      \
        }                                                         \
    } while (0)
    if (dir == 0) NS_GATED(0);
    else if (dir == 1) NS_GATED(1);
    else NS_GATED(2);
#undef NS_GATED
#undef NS_GATED1
    st->faces += (unsigned long long)fb.n0 * fb.n1 * fb.n2;
    if (launches) (*launches)++;
    return cudaGetLastError() == cudaSuccess ? NS_OK : NS_ERR_CUDA;
}

ns_status sensor_step_flags(SensorState* st, const double* U0, const Box& b, const Consts& c, double threshold,
                            const FaceBox fb[3], int conv_dims, cudaStream_t s, long long* launches) {
    const float thr = (float)std::log(threshold / (1.0 - threshold));
    const dim3 blk(32, 4);
    if (cudaMemsetAsync(st->counts, 0, 4 * sizeof(unsigned), s) != cudaSuccess ||
        cudaMemsetAsync(st->touched, 0, (size_t)st->ncells, s) != cudaSuccess)
        return NS_ERR_CUDA;
    // the step's rho, p, u, v, w in FP32, read by the three axes
    k_sensor_prims<<<dim3((b.nz + 31) / 32, (b.ny + 3) / 4, b.nx), blk, 0, s>>>(U0, b, c, st->prim);
    if (launches) (*launches)++;
    for (int d = 0; d < conv_dims; d++) {
        const FaceBox& f = fb[d];
        const long long tiles = (long long)((f.n2 + 31) / 32) * ((f.n1 + 3) / 4) * f.n0;
        if (tiles >= (1ll << 31) || f.fstride >= (1ll << 32)) return NS_ERR_UNSUPPORTED;
        const int grid = (int)std::min<long long>(tiles, (long long)st->sms * 8);
#define NS_MASK(D) k_sensor_mask_tc<D><<<grid, blk, 0, s>>>(st->prim, b, c, f, st->w, thr, st->mask[D], st->flagged, \
                                                          st->list[D], st->counts + D, st->touched, st->err)
        if (d == 0) NS_MASK(0);
        else if (d == 1) NS_MASK(1);
        else NS_MASK(2);
#undef NS_MASK
        st->faces += (unsigned long long)f.n0 * f.n1 * f.n2;
        if (launches) (*launches)++;
    }
    k_sensor_touched_list<<<(unsigned)((st->ncells + 127) / 128), 128, 0, s>>>(st->touched, st->ncells, st->cells,
                                                                              st->counts + 3);
    if (launches) (*launches)++;
    return cudaGetLastError() == cudaSuccess ? NS_OK : NS_ERR_CUDA;
}

ns_status sensor_status(SensorState* st) {
    int e = 0;
    if (cudaMemcpy(&e, st->err, sizeof e, cudaMemcpyDeviceToHost) != cudaSuccess) return NS_ERR_CUDA;
    return e ? NS_ERR_TIMEOUT : NS_OK;
}

GateLists sensor_gate_lists(const SensorState* st) {
    GateLists L;
    for (int d = 0; d < 3; d++) {
        L.face_list[d] = st->list[d];
        L.mask[d] = st->mask[d];
    }
    L.face_count = st->counts;
    L.cell_list = st->cells;
    L.cell_count = st->counts + 3;
    L.touched = st->touched;
    return L;
}


double sensor_last_fraction(SensorState* st) {
    if (!st || st->faces == 0) return 0.0;
    unsigned long long n = 0;
    if (cudaMemcpy(&n, st->flagged, sizeof n, cudaMemcpyDeviceToHost) != cudaSuccess) return 0.0;
    return (double)n / (double)st->faces;
}

ns_status sensor_harvest(int dir, bool borges, bool phys, const double* W, const double* U, const Box& b,
                         const Consts& c, const FaceBox& fb, long long base, double thr, float* feat,
                         float* label, cudaStream_t s) {
    dim3 grid((fb.n2 + 31) / 32, (fb.n1 + 3) / 4, fb.n0), blk(32, 4);
#define NS_HARV(D)                                                                                          \
    do {                                                                                                    \
        if (phys) {                                                                                         \
            if (borges) k_sensor_harvest<D, true, true><<<grid, blk, 0, s>>>(W, U, b, c, fb, base, thr, feat, label); \
            else k_sensor_harvest<D, false, true><<<grid, blk, 0, s>>>(W, U, b, c, fb, base, thr, feat, label);      \
        } else {                                                                                            \
            if (borges) k_sensor_harvest<D, true, false><<<grid, blk, 0, s>>>(W, U, b, c, fb, base, thr, feat, label); \
            else k_sensor_harvest<D, false, false><<<grid, blk, 0, s>>>(W, U, b, c, fb, base, thr, feat, label);      \
        }                                                                                                   \
    } while (0)
    if (dir == 0) NS_HARV(0);
    else if (dir == 1) NS_HARV(1);
    else NS_HARV(2);
#undef NS_HARV
    return cudaGetLastError() == cudaSuccess ? NS_OK : NS_ERR_CUDA;
}

}  // namespace nsb

// ===========================================================================
// C ABI (training and evaluation of the sensor network)

using namespace nsb;

namespace {

unsigned long long gcd_u64(unsigned long long a, unsigned long long b) {
    while (b) { unsigned long long t = a % b; a = b; b = t; }
    return a;
}

unsigned long long splitmix(unsigned long long& s) {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

size_t train_smem() { return sizeof(TrainSmem); }

}  // namespace

extern "C" {

NS_API ns_status ns_sensor_init(unsigned long long seed, float* w) {
    if (!w) return NS_ERR_INVALID_ARG;
    unsigned long long s = seed;
    auto uni = [&]() { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0; };
    memset(w, 0, SP * sizeof(float));
    // Glorot-uniform weights, zero biases
    double a1 = std::sqrt(6.0 / (SF + SH)), a2 = std::sqrt(6.0 / (SH + SH)), a3 = std::sqrt(6.0 / (SH + 1));
    for (int o = 0; o < SH; o++)
        for (int i = 0; i < SF; i++) w[OFF_W1 + o * 32 + i] = (float)(a1 * uni());
    for (int o = 0; o < SH; o++)
        for (int i = 0; i < SH; i++) w[OFF_W2 + o * 32 + i] = (float)(a2 * uni());
    for (int i = 0; i < SH; i++) w[OFF_W3 + i] = (float)(a3 * uni());
    return NS_OK;
}

NS_API ns_status ns_sensor_gradients(const float* feat, const float* label, int n, float pos_weight,
                                     const float* w, float* grad, float* loss, void* stream) {
    if (!feat || !label || !w || !grad || n <= 0) return NS_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    float *dw = nullptr, *dg = nullptr, *dl = nullptr;
    if (cudaMalloc(&dw, SP * sizeof(float)) != cudaSuccess || cudaMalloc(&dg, SP * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&dl, sizeof(float)) != cudaSuccess) {
        cudaFree(dw); cudaFree(dg); cudaFree(dl);
        cudaGetLastError();
        return NS_ERR_OOM;
    }
    cudaMemcpyAsync(dw, w, SP * sizeof(float), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(dg, 0, SP * sizeof(float), s);
    cudaMemsetAsync(dl, 0, sizeof(float), s);
    cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem());
    // identity order: a = 1, c = 0
    k_mlp_train<<<(n + 127) / 128, 128, train_smem(), s>>>(feat, label, n, 0, n, 1, 0, pos_weight,
                                                          1.f / n, dw, dg, dl);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        cudaMemcpyAsync(grad, dg, SP * sizeof(float), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(loss, dl, sizeof(float), cudaMemcpyDeviceToHost, s);
        e = cudaStreamSynchronize(s);
    }
    cudaFree(dw); cudaFree(dg); cudaFree(dl);
    return e == cudaSuccess ? NS_OK : NS_ERR_CUDA;
}

NS_API ns_status ns_sensor_train(const float* feat, const float* label, long long n, int epochs,
                                 int batch, float lr, float pos_weight, unsigned long long seed,
                                 float* w, float* epoch_loss, void* stream) {
    if (!feat || !label || !w || n <= 0 || epochs <= 0 || batch <= 0 || !(lr > 0.f))
        return NS_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    float *dw = nullptr, *dm = nullptr, *dv = nullptr, *dg = nullptr, *dl = nullptr;
    bool ok = cudaMalloc(&dw, SP * sizeof(float)) == cudaSuccess && cudaMalloc(&dm, SP * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&dv, SP * sizeof(float)) == cudaSuccess && cudaMalloc(&dg, SP * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&dl, (size_t)epochs * sizeof(float)) == cudaSuccess;
    if (!ok) {
        cudaFree(dw); cudaFree(dm); cudaFree(dv); cudaFree(dg); cudaFree(dl);
        cudaGetLastError();
        return NS_ERR_OOM;
    }
    cudaMemcpyAsync(dw, w, SP * sizeof(float), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(dm, 0, SP * sizeof(float), s);
    cudaMemsetAsync(dv, 0, SP * sizeof(float), s);
    cudaMemsetAsync(dg, 0, SP * sizeof(float), s);
    cudaMemsetAsync(dl, 0, (size_t)epochs * sizeof(float), s);
    cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem());
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    unsigned long long rs = seed, t = 0;
    const long long nb = (n + batch - 1) / batch;
    for (int ep = 0; ep < epochs; ep++) {
        // a fresh pseudo-random order of the samples each epoch: i -> (a i + c) mod n
        unsigned long long pa = 0, pc = splitmix(rs) % (unsigned long long)n;
        do { pa = (splitmix(rs) % (unsigned long long)n) | 1ULL; } while (gcd_u64(pa, (unsigned long long)n) != 1ULL);
        for (long long bi = 0; bi < nb; bi++) {
            long long start = bi * batch;
            int cnt = (int)((n - start) < batch ? (n - start) : batch);
            k_mlp_train<<<(cnt + 127) / 128, 128, train_smem(), s>>>(
                feat, label, n, start, cnt, pa, pc, pos_weight, 1.f / cnt, dw, dg, dl + ep);
            t++;
            float c1 = 1.f / (1.f - std::pow(b1, (float)t)), c2 = 1.f / (1.f - std::pow(b2, (float)t));
            k_adam<<<3, 1024, 0, s>>>(dw, dm, dv, dg, lr, b1, b2, eps, c1, c2);
        }
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        cudaMemcpyAsync(w, dw, SP * sizeof(float), cudaMemcpyDeviceToHost, s);
        if (epoch_loss) {
            std::vector<float> h(epochs);
            cudaMemcpyAsync(h.data(), dl, (size_t)epochs * sizeof(float), cudaMemcpyDeviceToHost, s);
            e = cudaStreamSynchronize(s);
            for (int ep = 0; ep < epochs; ep++) epoch_loss[ep] = h[ep] / (float)nb;
        } else {
            e = cudaStreamSynchronize(s);
        }
    }
    cudaFree(dw); cudaFree(dm); cudaFree(dv); cudaFree(dg); cudaFree(dl);
    return e == cudaSuccess ? NS_OK : NS_ERR_CUDA;
}

NS_API ns_status ns_sensor_predict(const float* feat, long long n, const float* w, float* logit,
                                   void* stream) {
    if (!feat || !w || !logit || n <= 0) return NS_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    float* dw = nullptr;
    if (cudaMalloc(&dw, SP * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return NS_ERR_OOM;
    }
    cudaMemcpyAsync(dw, w, SP * sizeof(float), cudaMemcpyHostToDevice, s);
    k_mlp_predict<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(feat, n, dw, logit);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(dw);
    return e == cudaSuccess ? NS_OK : NS_ERR_CUDA;
}

}  // extern "C"
