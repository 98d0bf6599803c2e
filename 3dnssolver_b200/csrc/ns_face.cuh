// ns_face.cuh -- WENO-5 face flux of one face (device functions).
//
// A face along axis DIR lies between cells a and a+1; its 6-cell stencil is
// a-2..a+3.  face_stencil loads the stencil, forms half the Euler flux of each
// cell and the Lax-Friedrichs split fL = (F + alpha U)/2 (cells a-2..a+2),
// fR = (F - alpha U)/2 (cells a-1..a+3); face_comp and face_char turn the split
// into the numerical flux component-wise (Weno5::x/y/z_sweep,
// src/convection_schemes/weno-5.cpp:75-220) or in characteristic variables
// (Weno5cw, src/convection_schemes/weno-5cw.cpp:4-262).
#pragma once

#include "ns_common.cuh"

namespace nsb {

// Tangent frame of ConvectionFlux::orthogonal_unit_vectors (convection_flux.cpp:63-115)
// for the axis normals: x: l = e_z, m = -e_y;  y: l = e_z, m = e_x;  z: l = -e_y, m = e_x.
template <int DIR>
struct Frame;
template <>
struct Frame<0> {
    static constexpr int l_ax = 2, l_sg = 1, m_ax = 1, m_sg = -1;
};
template <>
struct Frame<1> {
    static constexpr int l_ax = 2, l_sg = 1, m_ax = 0, m_sg = 1;
};
template <>
struct Frame<2> {
    static constexpr int l_ax = 1, l_sg = -1, m_ax = 0, m_sg = 1;
};

// State index of textbook component t of [rho, rho u, rho v, rho w, rho E].
// The reference applies its textbook-ordered eigenvectors to the state order
// [rho, rhoE, rhou, rhov, rhow] unchanged (convection_flux.cpp:153-171 vs
// src/domain.hpp:52), i.e. the identity map; the physical form permutes.
template <bool PHYS>
__device__ __forceinline__ constexpr int st(int t) {
    return PHYS ? (t == 0 ? 0 : (t == 4 ? 1 : t + 1)) : t;
}

template <typename T>
__device__ __forceinline__ T tsqrt(T x) {
    if constexpr (sizeof(T) == 8) return sqrt(x); else return sqrtf(x);
}
template <typename T>
__device__ __forceinline__ T trcp(T x) {
    if constexpr (sizeof(T) == 8) return 1.0 / x; else return __fdividef(1.0f, x);
}

// Left/right eigenvectors of the 3D Euler Jacobian (ConvectionFlux::eigenvectors,
// convection_flux.cpp:117-175) at the arithmetic face average, kept as the
// scalars the sparse rows need.
template <typename T>
struct Eig {
    T vel[3], qn, ql, qm, q2, c, c2, H, Kpc, K2pc, inv2c;
};

// 1/sqrt(x), x > 0 (sound speeds): Newton-Raphson in FP64 (rsqrt_pos_nr)
template <typename T>
__device__ __forceinline__ T trsqrt(T x) {
    if constexpr (sizeof(T) == 8) {
        if constexpr (NS_RSQRT_NR) return rsqrt_pos_nr(x);
        else return rsqrt(x);
    } else {
        return rsqrtf(x);
    }
}

// Reference semantics (c2 = gamma/(p rho), convection_flux.cpp:139): one
// r = rsqrt(p rho) and one rg = rsqrt(gamma) give c = sqrt(gamma) r,
// 1/(2c) = p rho r rg / 2 and K/(2 c2) = (gamma-1) p rho rg^2 / 2 without a
// division or square root.
template <int DIR, bool PHYS, typename T>
__device__ __forceinline__ Eig<T> make_eig(const T wa[5], T gamma, T inv_gm1) {
    Eig<T> e;
    T rho = wa[0], p = wa[1];
    e.vel[0] = wa[2]; e.vel[1] = wa[3]; e.vel[2] = wa[4];
    e.qn = e.vel[DIR];
    e.ql = Frame<DIR>::l_sg * e.vel[Frame<DIR>::l_ax];
    e.qm = Frame<DIR>::m_sg * e.vel[Frame<DIR>::m_ax];
    e.q2 = e.vel[0] * e.vel[0] + e.vel[1] * e.vel[1] + e.vel[2] * e.vel[2];
    T K = gamma - T(1);
    if constexpr (PHYS) {
        // c2 = gamma p / rho from one r = rsqrt(gamma p rho): c = gamma p r,
        // 1/c = rho r, so no division or square root (each costs a Newton
        // sequence in FP64)
        const T gp = gamma * p;
        const T r = trsqrt(gp * rho);
        const T ic = rho * r;
        e.c = gp * r;
        e.c2 = e.c * e.c;
        e.Kpc = K * T(0.5) * (ic * ic);
        e.inv2c = T(0.5) * ic;
    } else {
        T pr = p * rho;
        T r = trsqrt(pr);
        // sqrt(gamma) and 1/gamma from one rg = rsqrt(gamma): no square root or
        // division per face
        const T rg = trsqrt(gamma);
        e.c = (gamma * rg) * r;
        e.c2 = gamma * (r * r);
        e.Kpc = (K * T(0.5) * (rg * rg)) * pr;
        e.inv2c = (T(0.5) * rg) * (pr * r);
    }
    e.H = e.c2 * inv_gm1 + T(0.5) * e.q2;
    e.K2pc = T(2) * e.Kpc;  // K/c2
    return e;
}

// char_r = sum_t L[r][t] f[st(t)] for the textbook rows of L
template <int DIR, bool PHYS, int R, typename T>
__device__ __forceinline__ T lproj(const Eig<T>& e, const T f[5]) {
    const T f0 = f[st<PHYS>(0)];
    const T fe = f[st<PHYS>(4)];
    const T fm[3] = {f[st<PHYS>(1)], f[st<PHYS>(2)], f[st<PHYS>(3)]};
    if constexpr (R == 1) {  // (-qm, m, 0)
        constexpr int a = Frame<DIR>::m_ax;
        return -e.qm * f0 + (Frame<DIR>::m_sg > 0 ? fm[a] : -fm[a]);
    } else if constexpr (R == 4) {  // (-ql, l, 0)
        constexpr int a = Frame<DIR>::l_ax;
        return -e.ql * f0 + (Frame<DIR>::l_sg > 0 ? fm[a] : -fm[a]);
    } else if constexpr (R == 2) {  // (1 - Kpc q2, K u/c2, K v/c2, K w/c2, -K/c2)
        return (T(1) - e.Kpc * e.q2) * f0 + e.K2pc * (e.vel[0] * fm[0] + e.vel[1] * fm[1] + e.vel[2] * fm[2]) -
               e.K2pc * fe;
    } else {  // R == 0 (+) or R == 3 (-): (Kpc q2/2 +- qn/2c, -(Kpc u +- n_x/2c), ..., Kpc)
        constexpr T sg = (R == 0) ? T(1) : T(-1);
        T s = (T(0.5) * e.Kpc * e.q2 + sg * e.qn * e.inv2c) * f0 -
              e.Kpc * (e.vel[0] * fm[0] + e.vel[1] * fm[1] + e.vel[2] * fm[2]) + e.Kpc * fe;
        return s - sg * e.inv2c * fm[DIR];
    }
}

// halo'd offset of stencil cell 0 of face (aa, bb, kk) in face-box coordinates,
// and the stride between stencil cells
template <int DIR>
__device__ __forceinline__ long long face_origin(const Box& b, int aa, int bb, int kk, long long& step) {
    step = DIR == 0 ? (long long)b.NY * b.NZp : (DIR == 1 ? (long long)b.NZp : 1LL);
    int ih = aa + (DIR == 0 ? 0 : NG), jh = bb + (DIR == 1 ? 0 : NG), kh = kk + (DIR == 2 ? 0 : NG);
    return b.at(ih, jh, kh);
}

// Half the Euler flux of one cell along DIR (ConvectionFlux::form_flux,
// convection_flux.cpp:23-61): rho q_n H = q_n (gamma p/(gamma-1) + rho |u|^2/2)
// needs no division.  hg = gamma/(2(gamma-1)).
template <int DIR, typename T>
__device__ __forceinline__ void half_flux(const T w[5], T hg, T f[5]) {
    const T half = T(0.5);
    T rho = w[0], p = w[1];
    T qn = w[2 + DIR];
    T hrq = half * rho * qn;
    T ke = w[2] * w[2] + w[3] * w[3] + w[4] * w[4];
    f[0] = hrq;
    f[1] = qn * (hg * p + T(0.25) * rho * ke);
    f[2] = hrq * w[2] + (DIR == 0 ? half * p : T(0));
    f[3] = hrq * w[3] + (DIR == 1 ? half * p : T(0));
    f[4] = hrq * w[4] + (DIR == 2 ? half * p : T(0));
}

// Lax-Friedrichs split of stencil cell s with halpha = alpha/2 (reference
// semantics: alpha = 3): fL = (F + alpha U)/2 for s = 0..4, fR = (F - alpha U)/2
// for s = 1..5; the face average of W is taken from cells 2 and 3.
template <int DIR, bool CHAR, typename T>
__device__ __forceinline__ void split_cell(int s, const T w[5], const T u[5], T hg, T fL[5][5],
                                           T fR[5][5], T wa[5], T halpha = T(1.5)) {
    const T half = T(0.5);
    if constexpr (CHAR) {
        if (s == 2) {
#pragma unroll
            for (int q = 0; q < 5; q++) wa[q] = w[q];
        }
        if (s == 3) {
#pragma unroll
            for (int q = 0; q < 5; q++) wa[q] = half * (wa[q] + w[q]);
        }
    }
    T f[5];
    half_flux<DIR, T>(w, hg, f);
#pragma unroll
    for (int q = 0; q < 5; q++) {
        if (s <= 4) fL[q][s] = halpha * u[q] + f[q];
        if (s >= 1) fR[q][s - 1] = f[q] - halpha * u[q];
    }
}

// Euler flux + Lax-Friedrichs split of a 6-cell stencil whose cells the loader
// supplies: ld(s, w, u) gives W and U of stencil cell s; wa receives the face
// average of W (characteristic form only)
template <int DIR, bool CHAR, bool PHYS, typename T, typename Loader>
__device__ __forceinline__ void face_stencil_from(Loader ld, const Consts& c, T fL[5][5], T fR[5][5],
                                                  T wa[5]) {
    const T gamma = T(c.gamma), half = T(0.5);
    const T hg = half * gamma * T(c.inv_gm1);  // gamma/(2(gamma-1))
    if constexpr (!PHYS) {
#pragma unroll
        for (int s = 0; s < 6; s++) {
            T w[5], u[5];
            ld(s, w, u);
            split_cell<DIR, CHAR, T>(s, w, u, hg, fL, fR, wa);
        }
    } else {
        // local Lax-Friedrichs speed max(|q_n| + c) over the 6-cell stencil, in a first
        // pass over the stencil (the second pass reloads its cells from L1), with
        // c = sqrt(gamma p/rho) = gamma p rsqrt(gamma p rho)
        T amax = T(0);
#pragma unroll
        for (int s = 0; s < 6; s++) {
            T w[5], u[5];
            ld(s, w, u);
            const T gp = gamma * w[1];
            const T a = fabs(w[2 + DIR]) + gp * trsqrt(gp * w[0]);
            amax = (s == 0) ? a : (a > amax ? a : amax);
        }
        const T halpha = half * amax;
#pragma unroll
        for (int s = 0; s < 6; s++) {
            T w[5], u[5];
            ld(s, w, u);
            split_cell<DIR, CHAR, T>(s, w, u, hg, fL, fR, wa, halpha);
        }
    }
}

// stencil load from the device state + Euler flux + Lax-Friedrichs split
template <int DIR, bool CHAR, bool PHYS, typename T>
__device__ __forceinline__ void face_stencil(const double* __restrict__ W, const double* __restrict__ U,
                                             const Box& b, const Consts& c, long long o0,
                                             long long step, T fL[5][5], T fR[5][5], T wa[5]) {
    auto ld = [&](int s, T w[5], T u[5]) {
        const long long o = o0 + s * step;
#pragma unroll
        for (int q = 0; q < 5; q++) {
            w[q] = T(W[q * b.fstride + o]);
            u[q] = T(U[q * b.fstride + o]);
        }
    };
    face_stencil_from<DIR, CHAR, PHYS, T>(ld, c, fL, fR, wa);
}

// component-wise: f_q = WENO5_left(fL_q) + WENO5_right(fR_q)   (weno-5.cpp:96-114)
template <typename T, bool BORGES>
__device__ __forceinline__ void face_comp(const T fL[5][5], const T fR[5][5], T out[5]) {
#pragma unroll
    for (int q = 0; q < 5; q++)
        out[q] = weno_pair<T, BORGES>(fL[q][0], fL[q][1], fL[q][2], fL[q][3], fL[q][4],
                                      fR[q][0], fR[q][1], fR[q][2], fR[q][3], fR[q][4]);
}

// characteristic-wise: project fL, fR with L at the face average, WENO per
// characteristic field, back-project with R (Weno5cw::compute_num_flux)
template <int DIR, bool PHYS, typename T, bool BORGES>
__device__ __forceinline__ void face_char(const T fL[5][5], const T fR[5][5], const T wa[5], T gamma,
                                      T inv_gm1, T out[5]) {
    const T half = T(0.5);
    Eig<T> e = make_eig<DIR, PHYS, T>(wa, gamma, inv_gm1);
    T ft[5];
    // characteristic projection L fL, L fR per stencil column, WENO per field
    // (Weno5cw::compute_num_flux, weno-5cw.cpp:4-28)
#define NS_CHAR_FIELD(RR)                                                        \
    {                                                                        \
        T cl[5], cr[5];                                                      \
        _Pragma("unroll") for (int s = 0; s < 5; s++) {                      \
            T vl[5] = {fL[0][s], fL[1][s], fL[2][s], fL[3][s], fL[4][s]};    \
            T vr[5] = {fR[0][s], fR[1][s], fR[2][s], fR[3][s], fR[4][s]};    \
            cl[s] = lproj<DIR, PHYS, RR, T>(e, vl);                          \
            cr[s] = lproj<DIR, PHYS, RR, T>(e, vr);                          \
        }                                                                    \
        ft[RR] = weno_pair<T, BORGES>(cl[0], cl[1], cl[2], cl[3], cl[4],      \
                                      cr[0], cr[1], cr[2], cr[3], cr[4]);     \
    }
    NS_CHAR_FIELD(0)
    NS_CHAR_FIELD(1)
    NS_CHAR_FIELD(2)
    NS_CHAR_FIELD(3)
    NS_CHAR_FIELD(4)
#undef NS_CHAR_FIELD
    // back-projection R ft; textbook rows of R (convection_flux.cpp:153-158)
    T acc = ft[0] + ft[2] + ft[3];
    T tb[5];
    tb[0] = acc;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        T cn = (a == DIR) ? e.c : T(0);
        T v = e.vel[a] * acc - cn * ft[0] + cn * ft[3];
        if (a == Frame<DIR>::m_ax) v += (Frame<DIR>::m_sg > 0 ? ft[1] : -ft[1]);
        if (a == Frame<DIR>::l_ax) v += (Frame<DIR>::l_sg > 0 ? ft[4] : -ft[4]);
        tb[1 + a] = v;
    }
    tb[4] = e.H * (ft[0] + ft[3]) + e.qn * e.c * (ft[3] - ft[0]) + e.qm * ft[1] +
            half * e.q2 * ft[2] + e.ql * ft[4];
#pragma unroll
    for (int t = 0; t < 5; t++) out[st<PHYS>(t)] = tb[t];
}

}  // namespace nsb
