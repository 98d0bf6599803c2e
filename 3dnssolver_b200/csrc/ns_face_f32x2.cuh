// ns_face_f32x2.cuh -- one WENO-5 face in packed FP32 (sm_100 f32x2 FMA/MUL/ADD).
//
// The numerical flux of a face is WENO5_left(fL) + WENO5_right(fR)
// (src/convection_schemes/weno-5.cpp:96-114).  The right-biased reconstruction
// of cells a-1..a+3 equals the left-biased formula applied to the same cells in
// reverse order (candidates, smoothness indicators and linear weights map onto
// each other), so both run as the two lanes of one float2 stream:
//   lane x: fL of cells a-2, a-1, a, a+1, a+2
//   lane y: fR of cells a+3, a+2, a+1, a, a-1
// The characteristic projection (Weno5cw::compute_num_flux, weno-5cw.cpp:4-28)
// is linear, so the left and right columns of the same stencil position are
// projected together as well.  PHYS = false: the reference semantics (alpha = 3,
// c2 = gamma/(p rho), textbook rows applied to the state order,
// convection_flux.cpp:139,153-171,241); PHYS = true: the physical form (local
// alpha = max(|q_n| + c) over the 6-cell stencil, c2 = gamma p/rho, rows
// permuted to the state order).
#pragma once

#include "ns_face.cuh"

namespace nsb {

typedef float2 f2;

__device__ __forceinline__ f2 sp2(float a) { return make_float2(a, a); }
__device__ __forceinline__ f2 add2(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 mul2(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ f2 sub2(f2 a, f2 b) { return __ffma2_rn(sp2(-1.f), b, a); }  // exact a - b

// WENO-5 left-biased reconstruction (weno-5.cpp:305-322) on both lanes, summed:
// FP32 weights as in weno_weights<float> (epsilon raised to the stencil's
// rounding level), one fast reciprocal per weight and per lane.
template <bool BORGES>
__device__ __forceinline__ float weno_f32x2(f2 a, f2 b, f2 c, f2 d, f2 e) {
    const f2 k1312 = sp2(13.f / 12.f), k14 = sp2(0.25f);
    f2 t1 = fma2(sp2(-2.f), b, add2(a, c));
    f2 t2 = fma2(sp2(-4.f), b, fma2(sp2(3.f), c, a));
    f2 b0 = fma2(mul2(k1312, t1), t1, mul2(mul2(k14, t2), t2));
    t1 = fma2(sp2(-2.f), c, add2(b, d));
    t2 = sub2(b, d);
    f2 b1 = fma2(mul2(k1312, t1), t1, mul2(mul2(k14, t2), t2));
    t1 = fma2(sp2(-2.f), d, add2(c, e));
    t2 = fma2(sp2(-4.f), d, fma2(sp2(3.f), c, e));
    f2 b2 = fma2(mul2(k1312, t1), t1, mul2(mul2(k14, t2), t2));
    f2 n0, n1, n2;
    if constexpr (BORGES) {
        f2 tau = sub2(b0, b2);
        tau.x = fabsf(tau.x);
        tau.y = fabsf(tau.y);
        const f2 eb = sp2(WenoC<float>::eps_borges);
        f2 B0 = add2(b0, eb), B1 = add2(b1, eb), B2 = add2(b2, eb);
        n0 = make_float2(__fdividef(tau.x, B0.x), __fdividef(tau.y, B0.y));
        n1 = make_float2(__fdividef(tau.x, B1.x), __fdividef(tau.y, B1.y));
        n2 = make_float2(__fdividef(tau.x, B2.x), __fdividef(tau.y, B2.y));
        n0 = fma2(sp2(0.1f), n0, sp2(0.1f));
        n1 = fma2(sp2(0.6f), n1, sp2(0.6f));
        n2 = fma2(sp2(0.3f), n2, sp2(0.3f));
    } else {
        float sx = fmaxf(fmaxf(fmaxf(fabsf(a.x), fabsf(b.x)), fmaxf(fabsf(c.x), fabsf(d.x))), fabsf(e.x));
        float sy = fmaxf(fmaxf(fmaxf(fabsf(a.y), fabsf(b.y)), fmaxf(fabsf(c.y), fabsf(d.y))), fabsf(e.y));
        f2 fl = mul2(sp2(8.f * 5.9604645e-8f), make_float2(sx, sy));
        fl = mul2(fl, fl);
        f2 eps = make_float2(fmaxf(WenoC<float>::eps_shu, fl.x), fmaxf(WenoC<float>::eps_shu, fl.y));
        f2 s0 = add2(eps, b0), s1 = add2(eps, b1), s2 = add2(eps, b2);
        s0 = mul2(s0, s0);
        s1 = mul2(s1, s1);
        s2 = mul2(s2, s2);
        n0 = make_float2(__fdividef(0.1f, s0.x), __fdividef(0.1f, s0.y));
        n1 = make_float2(__fdividef(0.6f, s1.x), __fdividef(0.6f, s1.y));
        n2 = make_float2(__fdividef(0.3f, s2.x), __fdividef(0.3f, s2.y));
    }
    // ENO candidates at 6x their value (convection_constants.hpp coefficients)
    f2 f0 = fma2(sp2(11.f), c, fma2(sp2(-7.f), b, mul2(sp2(2.f), a)));
    f2 f1 = fma2(sp2(5.f), c, fma2(sp2(2.f), d, mul2(sp2(-1.f), b)));
    f2 fz = fma2(sp2(5.f), d, fma2(sp2(-1.f), e, mul2(sp2(2.f), c)));
    f2 num = fma2(n2, fz, fma2(n1, f1, mul2(n0, f0)));
    f2 den = mul2(sp2(6.f), add2(add2(n0, n1), n2));
    return __fdividef(num.x, den.x) + __fdividef(num.y, den.y);
}

// Half the Euler flux along DIR (half_flux) and U = cons(W) of two cells at once.
template <int DIR>
__device__ __forceinline__ void cell_pair_f32x2(const f2 w[5], float hg, float inv_gm1, f2 u[5], f2 f[5]) {
    const f2 half = sp2(0.5f);
    const f2 hr = mul2(half, w[0]);
    const f2 hrq = mul2(hr, w[2 + DIR]);
    const f2 ke = fma2(w[2], w[2], fma2(w[3], w[3], mul2(w[4], w[4])));
    u[0] = w[0];
    u[1] = fma2(w[1], sp2(inv_gm1), mul2(hr, ke));
    u[2] = mul2(w[0], w[2]);
    u[3] = mul2(w[0], w[3]);
    u[4] = mul2(w[0], w[4]);
    f[0] = hrq;
    f[1] = mul2(w[2 + DIR], fma2(sp2(hg), w[1], mul2(mul2(sp2(0.5f), hr), ke)));
    const f2 hp = mul2(half, w[1]);
    f[2] = DIR == 0 ? fma2(hrq, w[2], hp) : mul2(hrq, w[2]);
    f[3] = DIR == 1 ? fma2(hrq, w[3], hp) : mul2(hrq, w[3]);
    f[4] = DIR == 2 ? fma2(hrq, w[4], hp) : mul2(hrq, w[4]);
}

// Packed stencil of one face: P[q][k] = (fL_q of cell k, fR_q of cell 5-k),
// cells 0..5 = a-2..a+3, from W at the 6 cells: cells k and 5-k share a lane
// pair for U = cons(W) and half the Euler flux (division free); Lax-Friedrichs
// split with alpha = 3 (PHYS: the largest |q_n| + c of the 6 cells, c from one
// reciprocal square root: sqrt(gamma p/rho) = gamma p rsqrt(gamma p rho)).
// wa receives the face average of W (cells 2 and 3).
template <int DIR, bool CHAR, bool PHYS = false>
__device__ __forceinline__ void stencil_f32x2(const float* const* planes, int c0, int step, int fs,
                                              float gamma, float inv_gm1, f2 P[5][5], float wa[5]) {
    const float hg = 0.5f * gamma * inv_gm1;
    f2 U[3][5], F[3][5];
    float amax = 0.f;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float* A = planes[k];
        const float* B = planes[5 - k];
        const int ia = c0 + k * step, ib = c0 + (5 - k) * step;
        f2 w[5];
#pragma unroll
        for (int q = 0; q < 5; q++) w[q] = make_float2(A[q * fs + ia], B[q * fs + ib]);
        if constexpr (CHAR) {
            if (k == 2) {
#pragma unroll
                for (int q = 0; q < 5; q++) wa[q] = 0.5f * (w[q].x + w[q].y);
            }
        }
        if constexpr (PHYS) {
            const f2 gp = mul2(sp2(gamma), w[1]);
            const f2 gpr = mul2(gp, w[0]);
            const float cx = gp.x * rsqrtf(gpr.x), cy = gp.y * rsqrtf(gpr.y);
            amax = fmaxf(amax, fmaxf(fabsf(w[2 + DIR].x) + cx, fabsf(w[2 + DIR].y) + cy));
        }
        cell_pair_f32x2<DIR>(w, hg, inv_gm1, U[k], F[k]);
    }
    const float ha = PHYS ? 0.5f * amax : 1.5f;
    const f2 lr = make_float2(ha, -ha);
#pragma unroll
    for (int q = 0; q < 5; q++) {
#pragma unroll
        for (int k = 0; k < 3; k++) P[q][k] = fma2(lr, U[k][q], F[k][q]);
        // k = 3, 4: the pairs (2,3) and (1,4) with their lanes swapped
        P[q][3] = make_float2(fmaf(ha, U[2][q].y, F[2][q].y), fmaf(-ha, U[2][q].x, F[2][q].x));
        P[q][4] = make_float2(fmaf(ha, U[1][q].y, F[1][q].y), fmaf(-ha, U[1][q].x, F[1][q].x));
    }
}

template <int DIR, bool CHAR, bool BORGES, bool PHYS = false>
__device__ __forceinline__ void face_f32x2(const float* const* planes, int c0, int step, int fs, float gamma,
                                           float inv_gm1, float out[5]) {
    f2 P[5][5];
    float wa[5];
    stencil_f32x2<DIR, CHAR, PHYS>(planes, c0, step, fs, gamma, inv_gm1, P, wa);
    if constexpr (!CHAR) {
#pragma unroll
        for (int q = 0; q < 5; q++) out[q] = weno_f32x2<BORGES>(P[q][0], P[q][1], P[q][2], P[q][3], P[q][4]);
        return;
    } else {
        const Eig<float> e = make_eig<DIR, PHYS, float>(wa, gamma, inv_gm1);
        using F = Frame<DIR>;
        // state index of textbook component t (identity for the reference semantics)
        constexpr int s0 = st<PHYS>(0), s1 = st<PHYS>(1), s2 = st<PHYS>(2), s3 = st<PHYS>(3), s4 = st<PHYS>(4);
        // rows of L (make_eig's scalars); the tangential rows are kept up to
        // their sign (l_sg, m_sg): WENO is odd, so the sign is applied after it
        const f2 v0 = sp2(e.vel[0]), v1 = sp2(e.vel[1]), v2 = sp2(e.vel[2]);
        const f2 nqm = sp2(-F::m_sg * e.qm), nql = sp2(-F::l_sg * e.ql);
        const f2 r2a = sp2(1.f - e.Kpc * e.q2), k2 = sp2(e.K2pc), nk = sp2(-e.Kpc);
        const f2 a0 = sp2(0.5f * e.Kpc * e.q2 + e.qn * e.inv2c), a3 = sp2(0.5f * e.Kpc * e.q2 - e.qn * e.inv2c);
        const f2 i2c = sp2(e.inv2c);
        f2 C[5][5];
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const f2 f0 = P[s0][k], fe = P[s4][k];
            const f2 fm[3] = {P[s1][k], P[s2][k], P[s3][k]};
            f2 g = sub2(fma2(v0, fm[0], fma2(v1, fm[1], mul2(v2, fm[2]))), fe);  // u.fm - fE
            C[1][k] = fma2(nqm, f0, fm[F::m_ax]);                                 // m_sg * row 1
            C[4][k] = fma2(nql, f0, fm[F::l_ax]);                                 // l_sg * row 4
            C[2][k] = fma2(r2a, f0, mul2(k2, g));
            f2 kg = mul2(nk, g), ic = mul2(i2c, fm[DIR]);
            C[0][k] = fma2(a0, f0, sub2(kg, ic));
            C[3][k] = fma2(a3, f0, add2(kg, ic));
        }
        float ft[5];
#pragma unroll
        for (int r = 0; r < 5; r++) ft[r] = weno_f32x2<BORGES>(C[r][0], C[r][1], C[r][2], C[r][3], C[r][4]);
        ft[1] *= float(F::m_sg);
        ft[4] *= float(F::l_sg);
        // back-projection R ft (textbook rows of R, convection_flux.cpp:153-158)
        const float acc = ft[0] + ft[2] + ft[3];
        out[s0] = acc;
        constexpr int sm[3] = {s1, s2, s3};
#pragma unroll
        for (int ax = 0; ax < 3; ax++) {
            float cn = (ax == DIR) ? e.c : 0.f;
            float v = e.vel[ax] * acc - cn * ft[0] + cn * ft[3];
            if (ax == F::m_ax) v += (F::m_sg > 0 ? ft[1] : -ft[1]);
            if (ax == F::l_ax) v += (F::l_sg > 0 ? ft[4] : -ft[4]);
            out[sm[ax]] = v;
        }
        out[s4] = e.H * (ft[0] + ft[3]) + e.qn * e.c * (ft[3] - ft[0]) + e.qm * ft[1] + 0.5f * e.q2 * ft[2] +
                  e.ql * ft[4];
    }
}

}  // namespace nsb
