// ns_common.cuh -- device layout and shared device helpers.
//
// Device state layout (HBM): structure of arrays, one plane per variable,
// each plane the halo'd box (nx+6) x (ny+6) x NZp doubles with k fastest.
// NZp = nz+6 rounded up to 8, and the plane stride (fstride) a multiple of 8
// doubles, so every plane and every k-row starts on a 64-byte boundary (the
// TMA tensor maps of the FP64 face kernels need 16-byte row strides).
// Halos are real storage: the boundary fill writes them (the single-GPU form
// of Domain::apply_boundary_conditions + Communicator::communicate), and the
// per-operator entry points accept a caller's halos verbatim.
#pragma once

#include <cstdint>

#include "../../include/ns_b200.h"

#define NS_HOST_DEVICE __host__ __device__ __forceinline__

namespace nsb {

constexpr int NG = 3;
constexpr int NQV = 5;
constexpr int PLANE_PAD = 5;  // spare elements at the end of every plane

struct Box {
    int nx, ny, nz;     // interior cells
    int NX, NY, NZp;    // halo'd extents (NZp padded)
    long long fstride;  // elements per variable plane (incl. alignment pad)

    NS_HOST_DEVICE long long at(int ih, int jh, int kh) const {
        return ((long long)ih * NY + jh) * NZp + kh;
    }
};

inline Box make_box(int nx, int ny, int nz) {
    Box b;
    b.nx = nx; b.ny = ny; b.nz = nz;
    b.NX = nx + 2 * NG; b.NY = ny + 2 * NG;
    b.NZp = ((nz + 2 * NG + 7) / 8) * 8;
    long long plane = (long long)b.NX * b.NY * b.NZp;
    b.fstride = ((plane + PLANE_PAD + 7) / 8) * 8;
    return b;
}

// Face arrays: one plane per variable of (n_d+1) faces along the sweep axis,
// interior extent in the other two, k fastest.  Face f along an axis lies
// between interior cells f-1 and f.
struct FaceBox {
    int n0, n1, n2;     // extents (i or face, j or face, k or face)
    long long fstride;
    NS_HOST_DEVICE long long at(int a, int b, int c) const {
        return ((long long)a * n1 + b) * n2 + c;
    }
};

inline FaceBox make_facebox(int nx, int ny, int nz, int dir) {
    FaceBox f;
    f.n0 = nx + (dir == 0);
    f.n1 = ny + (dir == 1);
    f.n2 = nz + (dir == 2);
    f.fstride = (((long long)f.n0 * f.n1 * f.n2 + 31) / 32) * 32;
    return f;
}

// Kernel-side constants derived from ns_params.
struct Consts {
    double gamma, gm1, inv_gm1;
    double mu, lamb, heat;      // lamb = -2/3 mu, heat = gamma/(Pr(gamma-1))
    double dx, dy, dz, inv_dx, inv_dy, inv_dz;
    double cfl;
    int periodic[3];
    int dim;
    int order;                  // CD order 2/4/6
    double df[7], ddf[7];       // CD coefficients, centred at index 3
    // slab of a domain split along x (NS_BC_EXTERNAL): the x ghost planes hold the
    // neighbouring slabs' cells; x0 = global index of interior cell 0, nxg = global
    // cells along x, xper = global x axis periodic
    int ext_x, x0, nxg, xper;
};

#ifdef __CUDACC__
// 8-byte asynchronous global -> shared copies (cp.async, completion per thread)
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
#endif

// Periodic wrap or Neumann clamp of an interior-coordinate index.
NS_HOST_DEVICE int fold(int i, int n, int periodic) {
    if (i >= 0 && i < n) return i;
    if (periodic) {
        int r = i % n;
        return r < 0 ? r + n : r;
    }
    return i < 0 ? 0 : n - 1;
}

// Whether column i (interior coordinate) lies inside the global domain along x or
// the global x axis is periodic: the reference's derivative ghost cells are zero
// outside (centered_diffusion.cpp:22-24 fills them only by communication).
NS_HOST_DEVICE bool x_inside(int i, int nx, const Consts& c) {
    if (c.ext_x) {
        const int g = i + c.x0;
        return (g >= 0 && g < c.nxg) || c.xper;
    }
    return (i >= 0 && i < nx) || c.periodic[0];
}

// Whether the lower (hi = 0) or upper (hi = 1) x ghost planes of a slab come from
// a neighbour (exchanged) rather than from this slab's own Neumann copy.
NS_HOST_DEVICE bool x_exchanged(int hi, int nx, const Consts& c) {
    if (!c.ext_x) return false;
    if (c.xper) return true;
    return hi ? (c.x0 + nx < c.nxg) : (c.x0 > 0);
}

// x index of a stencil cell outside the interior along x: folded like fold() on
// a single domain; on a slab an exchanged side's ghost planes hold the
// neighbour's cells, so the index is used as it is, and a side at a
// non-periodic global end folds like Neumann (its ghost planes are copies of
// the first interior plane).
NS_HOST_DEVICE int fold_x(int i, int nx, const Consts& c) {
    if (!c.ext_x) return fold(i, nx, c.periodic[0]);
    if (i < 0 && !x_exchanged(0, nx, c)) return 0;
    if (i >= nx && !x_exchanged(1, nx, c)) return nx - 1;
    return i;
}

// ---------------------------------------------------------------------------
// WENO-5 (Jiang-Shu smoothness indicators, src/convection_schemes/weno-5.cpp:222-322)
//
// The three nonlinear weights are formed without a division each: with
// s_k = eps + beta_k (Shu) the weights d_k/s_k^2 normalised by their sum equal
// d_k * prod_{j!=k} s_j^2 / sum_m d_m prod_{j!=m} s_j^2 (Borges: d_k (B_k+tau) prod_{j!=k} B_j),
// and the left and right reconstructions of one face share one division.
// The algebra is exact; results differ from the reference's form by rounding only.  Single precision keeps per-weight reciprocals
// (products of squares would leave the float range) and raises eps above the
// float rounding floor of beta: eps32 = max(eps, (8 u32 s)^2), s the largest
// |f| of the stencil.

template <typename T>
struct WenoC;
template <>
struct WenoC<double> {
    static constexpr double eps_shu = 1e-6, eps_borges = 1e-14;
};
template <>
struct WenoC<float> {
    static constexpr float eps_shu = 1e-6f, eps_borges = 1e-14f;
};

template <typename T>
__device__ __forceinline__ void weno_betas(T a, T b, T c, T d, T e, T& b0, T& b1, T& b2) {
    const T k1312 = T(13) / T(12), k14 = T(0.25);
    T t1 = a - T(2) * b + c, t2 = a - T(4) * b + T(3) * c;
    b0 = k1312 * t1 * t1 + k14 * t2 * t2;
    t1 = b - T(2) * c + d;
    t2 = b - d;
    b1 = k1312 * t1 * t1 + k14 * t2 * t2;
    t1 = c - T(2) * d + e;
    t2 = T(3) * c - T(4) * d + e;
    b2 = k1312 * t1 * t1 + k14 * t2 * t2;
}

// Weights of one reconstruction from the stencil (a..e) and linear weights
// (d0,d1,d2): n_k proportional to the nonlinear weights, with the common
// factor left in (exact algebra, see above).
template <typename T, bool BORGES>
__device__ __forceinline__ void weno_weights(T a, T b, T c, T d, T e, T d0, T d1, T d2, T& n0, T& n1,
                                             T& n2) {
    T b0, b1, b2;
    weno_betas(a, b, c, d, e, b0, b1, b2);
    if constexpr (sizeof(T) == 8) {
        if constexpr (BORGES) {
            T tau = fabs(b0 - b2);
            T B0 = b0 + WenoC<T>::eps_borges, B1 = b1 + WenoC<T>::eps_borges,
              B2 = b2 + WenoC<T>::eps_borges;
            n0 = d0 * (B0 + tau) * (B1 * B2);
            n1 = d1 * (B1 + tau) * (B0 * B2);
            n2 = d2 * (B2 + tau) * (B0 * B1);
        } else {
            T s0 = WenoC<T>::eps_shu + b0, s1 = WenoC<T>::eps_shu + b1, s2 = WenoC<T>::eps_shu + b2;
            T A0 = s0 * s0, A1 = s1 * s1, A2 = s2 * s2;
            n0 = d0 * (A1 * A2);
            n1 = d1 * (A0 * A2);
            n2 = d2 * (A0 * A1);
        }
    } else {
        if constexpr (BORGES) {
            T tau = fabsf(b0 - b2);
            n0 = d0 * (T(1) + __fdividef(tau, b0 + WenoC<T>::eps_borges));
            n1 = d1 * (T(1) + __fdividef(tau, b1 + WenoC<T>::eps_borges));
            n2 = d2 * (T(1) + __fdividef(tau, b2 + WenoC<T>::eps_borges));
        } else {
            T s = fmaxf(fmaxf(fmaxf(fabsf(a), fabsf(b)), fmaxf(fabsf(c), fabsf(d))), fabsf(e));
            T fl = T(8) * T(5.9604645e-8) * s;
            T eps = fmaxf(WenoC<T>::eps_shu, fl * fl);
            T s0 = eps + b0, s1 = eps + b1, s2 = eps + b2;
            n0 = __fdividef(d0, s0 * s0);
            n1 = __fdividef(d1, s1 * s1);
            n2 = __fdividef(d2, s2 * s2);
        }
    }
}

// WENO5_left (weno-5.cpp:305-322) as num/den: value at i+1/2 from the
// left-biased stencil a..e = i-2..i+2.  The ENO candidates are kept at 6x
// their value and the 1/6 goes into den.
template <typename T, bool BORGES>
__device__ __forceinline__ void weno_left_nd(T a, T b, T c, T d, T e, T& num, T& den) {
    T f0 = T(2) * a - T(7) * b + T(11) * c;
    T f1 = -b + T(5) * c + T(2) * d;
    T f2 = T(2) * c + T(5) * d - e;
    T n0, n1, n2;
    weno_weights<T, BORGES>(a, b, c, d, e, T(0.1), T(0.6), T(0.3), n0, n1, n2);
    num = n0 * f0 + n1 * f1 + n2 * f2;
    den = T(6) * (n0 + n1 + n2);
}

// WENO5_right (weno-5.cpp:285-303) as num/den: value at i+1/2 from the
// right-biased stencil a..e = i-1..i+3.
template <typename T, bool BORGES>
__device__ __forceinline__ void weno_right_nd(T a, T b, T c, T d, T e, T& num, T& den) {
    T f0 = -a + T(5) * b + T(2) * c;
    T f1 = T(2) * b + T(5) * c - d;
    T f2 = T(11) * c - T(7) * d + T(2) * e;
    T n0, n1, n2;
    weno_weights<T, BORGES>(a, b, c, d, e, T(0.3), T(0.6), T(0.1), n0, n1, n2);
    num = n0 * f0 + n1 * f1 + n2 * f2;
    den = T(6) * (n0 + n1 + n2);
}

// x / d for a positive, normal d (the WENO denominators: sums of products of
// squared smoothness indicators, each at least the epsilon): the reciprocal by
// two Newton-Raphson iterations y <- y + y (1 - d y) from the hardware estimate
// (PTX rcp.approx.ftz.f64), then the quotient with one Markstein correction
// (P. Markstein, IA-64 and Elementary Functions, 2000): q = x y, r = x - d q,
// q + r y.  Within an ulp of the rounded quotient.
#ifndef NS_WENO_NR
#define NS_WENO_NR 1
#endif
__device__ __forceinline__ double div_pos_nr(double x, double d) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    double e = fma(-d, y, 1.0);
    y = fma(y, e, y);
    e = fma(-d, y, 1.0);
    y = fma(y, e, y);
    const double q = x * y;
    const double r = fma(-d, q, x);
    return fma(r, y, q);
}

// 1 / sqrt(x) for a positive, normal x: two Newton-Raphson iterations
// y <- y + (y / 2)(1 - x y^2) from the hardware estimate (PTX
// rsqrt.approx.ftz.f64).  Within an ulp or two of the rounded value.
#ifndef NS_RSQRT_NR
#define NS_RSQRT_NR 1
#endif
__device__ __forceinline__ double rsqrt_pos_nr(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x * y, y, 1.0);
    y = fma(0.5 * y, e, y);
    e = fma(-x * y, y, 1.0);
    return fma(0.5 * y, e, y);
}

// f = WENO5_left(l) + WENO5_right(r) with one division in FP64:
// nL/dL + nR/dR = (nL dR + nR dL)/(dL dR); FP32 uses two fast reciprocals.
template <typename T, bool BORGES>
__device__ __forceinline__ T weno_pair(T l0, T l1, T l2, T l3, T l4, T r0, T r1, T r2, T r3, T r4) {
    T nL, dL, nR, dR;
    weno_left_nd<T, BORGES>(l0, l1, l2, l3, l4, nL, dL);
    weno_right_nd<T, BORGES>(r0, r1, r2, r3, r4, nR, dR);
    if constexpr (sizeof(T) == 8) {
        if constexpr (NS_WENO_NR) return div_pos_nr(nL * dR + nR * dL, dL * dR);
        else return (nL * dR + nR * dL) / (dL * dR);
    }
    else
        return __fdividef(nL, dL) + __fdividef(nR, dR);
}

}  // namespace nsb
