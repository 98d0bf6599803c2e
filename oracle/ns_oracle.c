/*
 * ns_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * Plain-C restatement of the reference hot path of hamsteri15/3DNSsolver:
 * equation of state, boundary fill, periodic halo exchange, WENO-5
 * component-wise and characteristic-wise convection with Lax-Friedrichs flux
 * splitting, centered diffusion, CFL time step and the SSP-RK3 step.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker; the product path never calls it.
 *
 * Arrays use the reference container layout (src/containers/array_4d.hpp:64-71):
 * AoS [i][j][k][q] with 3 ghost cells per side.  Every floating-point
 * expression keeps the reference's operation order, so a build with
 * -O2 -fno-fast-math -ffp-contract=off agrees bit-for-bit with the reference
 * compiled the same way (pinned by tests/test_oracle_golden.py against the
 * reference build in oracle/_ref and the fixtures in tests/golden/).
 *
 * NS_SEM_PHYSICAL switches each non-textbook term of the reference to the
 * textbook form; it has no reference counterpart (parity unpinned for it).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../include/ns_b200.h"

#define NG 3
#define NQ 5

typedef struct {
    int nx, ny, nz, NX, NY, NZ;
    double dx, dy, dz;
    /* slab of a domain split along x (bc[0] = NS_BC_EXTERNAL): whether the lower
     * and upper x ghost planes come from a neighbour, and the x range of planes
     * whose y/z ghost rows and y-derivatives are formed (the interior, plus
     * exchanged ghost planes) */
    int ext, exlo, exhi, xlo, xhi;
} geom;

static geom make_geom(const ns_params* p) {
    geom g;
    g.nx = p->nx; g.ny = p->ny; g.nz = p->nz;
    g.NX = p->nx + 2 * NG; g.NY = p->ny + 2 * NG; g.NZ = p->nz + 2 * NG;
    g.ext = p->bc[0] == NS_BC_EXTERNAL;
    g.exlo = g.ext && (p->slab_periodic || p->slab_x0 > 0);
    g.exhi = g.ext && (p->slab_periodic || p->slab_x0 + p->nx < p->slab_nx);
    g.xlo = g.exlo ? 0 : NG;
    g.xhi = p->nx + NG + (g.exhi ? NG : 0);
    /* src/grid.cpp:12-19 */
    g.dx = p->Lx / p->nx; g.dy = p->Ly / p->ny; g.dz = p->Lz / p->nz;
    return g;
}

static inline size_t IX(const geom* g, int i, int j, int k, int q) {
    return ((((size_t)i * g->NY) + (size_t)j) * g->NZ + (size_t)k) * NQ + (size_t)q;
}

static size_t n_all(const geom* g) { return (size_t)g->NX * g->NY * g->NZ * NQ; }

static double* zeros(const geom* g) { return (double*)calloc(n_all(g), sizeof(double)); }

static inline double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */
static inline double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */

/* ------------------------------------------------------------------------ */
/* Equation of state: src/eq_of_state.cpp:32-59, 61-87 (all cells incl. halos) */

static void prim_to_cons(const ns_params* p, const geom* g, const double* W, double* U) {
    const double gm = p->gamma;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < g->NX; i++)
        for (int j = 0; j < g->NY; j++)
            for (int k = 0; k < g->NZ; k++) {
                const double* w = W + IX(g, i, j, k, 0);
                double* u = U + IX(g, i, j, k, 0);
                u[0] = w[0];
                u[2] = w[0] * w[2];
                u[3] = w[0] * w[3];
                u[4] = w[0] * w[4];
                double kin = 0.5 * w[0] * (w[2] * w[2] + w[3] * w[3] + w[4] * w[4]);
                u[1] = w[1] / (gm - 1.0) + kin;
            }
}

static void cons_to_prim(const ns_params* p, const geom* g, const double* U, double* W) {
    const double gm = p->gamma;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < g->NX; i++)
        for (int j = 0; j < g->NY; j++)
            for (int k = 0; k < g->NZ; k++) {
                const double* u = U + IX(g, i, j, k, 0);
                double* w = W + IX(g, i, j, k, 0);
                w[0] = u[0];
                w[2] = u[2] / u[0];
                w[3] = u[3] / u[0];
                w[4] = u[4] / u[0];
                double kin = 0.5 * (w[2] * w[2] + w[3] * w[3] + w[4] * w[4]);
                w[1] = (gm - 1.0) * (u[1] - u[0] * kin);
            }
}

/* ------------------------------------------------------------------------ */
/* Boundary fill: Neumann zeroth-order copy on the face region of a
 * non-periodic axis (src/boundary_conditions/boundary_neumann.cpp:22-132,
 * src/domain.cpp:18-28), then the periodic face exchange of a single rank
 * (src/communicator.cpp:6-143 with the slices of src/containers/array_4d.cpp:39-164).
 * The exchange gathers the send slice before writing the receive slice, as
 * MPI_Sendrecv does. */

static void neumann_fill(const ns_params* p, const geom* g, double* A) {
    /* a slab fills only the x sides at a non-periodic global end */
    const int xlo_fill = p->bc[0] == NS_BC_NEUMANN || (g->ext && !g->exlo);
    const int xhi_fill = p->bc[0] == NS_BC_NEUMANN || (g->ext && !g->exhi);
    if (xlo_fill || xhi_fill) {
        for (int i = 0; i < NG; i++)
            for (int j = NG; j < g->ny + NG; j++)
                for (int k = NG; k < g->nz + NG; k++)
                    for (int q = 0; q < NQ; q++) {
                        if (xlo_fill) A[IX(g, i, j, k, q)] = A[IX(g, NG, j, k, q)];
                        if (xhi_fill) A[IX(g, g->nx + NG + i, j, k, q)] = A[IX(g, g->nx + NG - 1, j, k, q)];
                    }
    }
    if (p->bc[1] == NS_BC_NEUMANN) {
        for (int i = g->xlo; i < g->xhi; i++)
            for (int j = 0; j < NG; j++)
                for (int k = NG; k < g->nz + NG; k++)
                    for (int q = 0; q < NQ; q++) {
                        A[IX(g, i, j, k, q)] = A[IX(g, i, NG, k, q)];
                        A[IX(g, i, g->ny + NG + j, k, q)] = A[IX(g, i, g->ny + NG - 1, k, q)];
                    }
    }
    if (p->bc[2] == NS_BC_NEUMANN) {
        for (int i = g->xlo; i < g->xhi; i++)
            for (int j = NG; j < g->ny + NG; j++)
                for (int k = 0; k < NG; k++)
                    for (int q = 0; q < NQ; q++) {
                        A[IX(g, i, j, k, q)] = A[IX(g, i, j, NG, q)];
                        A[IX(g, i, j, g->nz + NG + k, q)] = A[IX(g, i, j, g->nz + NG - 1, q)];
                    }
    }
}

/* copy the face slab [lo, lo+3) of axis `ax` to [dst, dst+3), other axes interior
 * (along x: the planes xlo..xhi-1, which include a slab's exchanged ghost planes) */
static void slab_copy(const geom* g, double* A, int ax, int src, int dst) {
    int n0 = (ax == 0) ? NG : g->xhi - g->xlo, n1 = (ax == 1) ? NG : g->ny, n2 = (ax == 2) ? NG : g->nz;
    size_t cnt = (size_t)n0 * n1 * n2 * NQ, c = 0;
    double* buf = (double*)malloc(cnt * sizeof(double));
    for (int a = 0; a < n0; a++)
        for (int b = 0; b < n1; b++)
            for (int d = 0; d < n2; d++) {
                int i = (ax == 0) ? src + a : g->xlo + a;
                int j = (ax == 1) ? src + b : NG + b;
                int k = (ax == 2) ? src + d : NG + d;
                for (int q = 0; q < NQ; q++) buf[c++] = A[IX(g, i, j, k, q)];
            }
    c = 0;
    for (int a = 0; a < n0; a++)
        for (int b = 0; b < n1; b++)
            for (int d = 0; d < n2; d++) {
                int i = (ax == 0) ? dst + a : g->xlo + a;
                int j = (ax == 1) ? dst + b : NG + b;
                int k = (ax == 2) ? dst + d : NG + d;
                for (int q = 0; q < NQ; q++) A[IX(g, i, j, k, q)] = buf[c++];
            }
    free(buf);
}

static void communicate(const ns_params* p, const geom* g, double* A) {
    const int n[3] = {g->nx, g->ny, g->nz};
    for (int ax = 0; ax < 3; ax++) {
        /* MPI_PROC_NULL: no-op; a slab's x ghost planes come from the exchange */
        if (p->bc[ax] != NS_BC_PERIODIC) continue;
        slab_copy(g, A, ax, n[ax], 0);        /* "east to east": arr(n) -> arr(0) */
        slab_copy(g, A, ax, NG, NG + n[ax]);  /* "west to west": arr(ngc) -> arr(ngc+n) */
    }
}

/* ------------------------------------------------------------------------ */
/* WENO-5 reconstruction: src/convection_schemes/weno-5.cpp:222-322,
 * constants src/convection_schemes/convection_constants.hpp:4-12 */

static const double eps_shu = 1E-6;
static const double eps_borges = 1E-14;
static const double c16 = 1. / 6.;
static const double c1312 = 13. / 12.;
static const double c14 = 1. / 4.;
static const double d_left[3] = {0.1, 0.6, 0.3};
static const double d_right[3] = {0.3, 0.6, 0.1};

static void weno_weights(int borges, double a, double b, double c, double d, double e,
                         const double dk[3], double w[3]) {
    double t1, t2, b0, b1, b2;
    t1 = a - 2. * b + c;
    t2 = a - 4. * b + 3. * c;
    b0 = c1312 * t1 * t1 + c14 * t2 * t2;
    t1 = b - 2. * c + d;
    t2 = b - d;
    b1 = c1312 * t1 * t1 + c14 * t2 * t2;
    t1 = c - 2. * d + e;
    t2 = 3. * c - 4. * d + e;
    b2 = c1312 * t1 * t1 + c14 * t2 * t2;
    double a0, a1, a2;
    if (borges) {
        double tau5 = fabs(b0 - b2);
        a0 = dk[0] * (1.0 + (tau5 / (b0 + eps_borges)));
        a1 = dk[1] * (1.0 + (tau5 / (b1 + eps_borges)));
        a2 = dk[2] * (1.0 + (tau5 / (b2 + eps_borges)));
    } else {
        a0 = dk[0] / ((eps_shu + b0) * (eps_shu + b0));
        a1 = dk[1] / ((eps_shu + b1) * (eps_shu + b1));
        a2 = dk[2] / ((eps_shu + b2) * (eps_shu + b2));
    }
    double s = a0 + a1 + a2;
    w[0] = a0 / s; w[1] = a1 / s; w[2] = a2 / s;
}

static double weno_left(int borges, double a, double b, double c, double d, double e) {
    double f0 = (2. * a - 7. * b + 11. * c) * c16;
    double f1 = (-b + 5. * c + 2. * d) * c16;
    double f2 = (2. * c + 5. * d - e) * c16;
    double w[3];
    weno_weights(borges, a, b, c, d, e, d_left, w);
    return w[0] * f0 + w[1] * f1 + w[2] * f2;
}

static double weno_right(int borges, double a, double b, double c, double d, double e) {
    double f0 = (-a + 5. * b + 2. * c) * c16;
    double f1 = (2. * b + 5. * c - d) * c16;
    double f2 = (11. * c - 7. * d + 2. * e) * c16;
    double w[3];
    weno_weights(borges, a, b, c, d, e, d_right, w);
    return w[0] * f0 + w[1] * f1 + w[2] * f2;
}

/* ------------------------------------------------------------------------ */
/* Euler flux and eigensystem: src/convection_schemes/convection_flux.cpp */

/* ConvectionFlux::form_flux, convection_flux.cpp:23-61 (all cells) */
static void form_flux(const ns_params* p, const geom* g, const double* W, const double n[3],
                      double* F) {
    const double gm = p->gamma;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < g->NX; i++)
        for (int j = 0; j < g->NY; j++)
            for (int k = 0; k < g->NZ; k++) {
                const double* w = W + IX(g, i, j, k, 0);
                double* f = F + IX(g, i, j, k, 0);
                double rho = w[0], pr = w[1], u = w[2], v = w[3], ww = w[4];
                double qn = u * n[0] + v * n[1] + ww * n[2];
                double c = sqrt(gm * pr / rho);
                double H = c * c / (gm - 1.0) + 0.5 * (u * u + v * v + ww * ww);
                f[0] = rho * qn;
                f[1] = rho * qn * H;
                f[2] = rho * qn * u + pr * n[0];
                f[3] = rho * qn * v + pr * n[1];
                f[4] = rho * qn * ww + pr * n[2];
            }
}

/* ConvectionFlux::orthogonal_unit_vectors, convection_flux.cpp:63-115 */
static void orthogonal_unit_vectors(const double n[3], double l[3], double m[3]) {
    double nx = n[0], ny = n[1], nz = n[2];
    double tx = ny * ny + nz * nz, ty = nz * nz + nx * nx, tz = nx * nx + ny * ny;
    double lx = 0, ly = 0, lz = 0;
    if (tx >= ty && tx >= tz) { lx = 0.0; ly = -nz; lz = ny; }
    else if (ty >= tx && ty >= tz) { lx = -nz; ly = 0.0; lz = nx; }
    else if (tz >= tx && tz >= ty) { lx = -ny; ly = nx; lz = 0.0; }
    double t = sqrt(lx * lx + ly * ly + lz * lz);
    lx = lx / t; ly = ly / t; lz = lz / t;
    double mx = ny * lz - nz * ly, my = nz * lx - nx * lz, mz = nx * ly - ny * lx;
    double a = sqrt(mx * mx + my * my + mz * mz);
    l[0] = lx; l[1] = ly; l[2] = lz;
    m[0] = mx / a; m[1] = my / a; m[2] = mz / a;
}

/* ConvectionFlux::eigenvectors, convection_flux.cpp:117-175.
 * Reference semantics keep c2 = gamma/(p rho) (:139) and the [rho,rhou,rhov,rhow,rhoE]
 * row/column order applied to [rho,rhoE,rhou,rhov,rhow] state vectors (:153-171).
 * Physical semantics use c2 = gamma p / rho and permute L's columns / R's rows
 * to the state order. */
static void eigenvectors(int phys, double rho, double pr, double u, double v, double w,
                         double gm, const double n[3], const double l[3], const double m[3],
                         double L[5][5], double R[5][5]) {
    double nx = n[0], ny = n[1], nz = n[2], lx = l[0], ly = l[1], lz = l[2];
    double mx = m[0], my = m[1], mz = m[2];
    double c2 = phys ? gm * pr / rho : gm / (pr * rho);
    double c = sqrt(c2);
    double qn = u * nx + v * ny + w * nz;
    double ql = u * lx + v * ly + w * lz;
    double qm = u * mx + v * my + w * mz;
    double q2 = u * u + v * v + w * w;
    double H = c2 / (gm - 1.0) + 0.5 * q2;
    double K = gm - 1.0;
    double Kpc = K / (2.0 * c2);
    double RR[5][5] = {{1.0, 0.0, 1.0, 1.0, 0.0},
                       {u - c * nx, mx, u, u + c * nx, lx},
                       {v - c * ny, my, v, v + c * ny, ly},
                       {w - c * nz, mz, w, w + c * nz, lz},
                       {H - qn * c, qm, 0.5 * q2, H + qn * c, ql}};
    double LL[5][5] = {{0.5 * Kpc * q2 + qn / (2.0 * c), -(Kpc * u + nx / (2.0 * c)),
                        -(Kpc * v + ny / (2.0 * c)), -(Kpc * w + nz / (2.0 * c)), Kpc},
                       {-qm, mx, my, mz, 0.0},
                       {1.0 - Kpc * q2, K * u / c2, K * v / c2, K * w / c2, -K / c2},
                       {0.5 * Kpc * q2 - qn / (2.0 * c), -(Kpc * u - nx / (2.0 * c)),
                        -(Kpc * v - ny / (2.0 * c)), -(Kpc * w - nz / (2.0 * c)), Kpc},
                       {-ql, lx, ly, lz, 0.0}};
    if (!phys) {
        memcpy(R, RR, sizeof(RR));
        memcpy(L, LL, sizeof(LL));
    } else {
        /* state index -> textbook index: rho->0, rhoE->4, rhou->1, rhov->2, rhow->3 */
        static const int perm[5] = {0, 4, 1, 2, 3};
        for (int a = 0; a < 5; a++)
            for (int b = 0; b < 5; b++) {
                L[a][b] = LL[a][perm[b]];
                R[a][b] = RR[perm[a]][b];
            }
    }
}

/* local max |q_n| + c used by the physical semantics' Lax-Friedrichs alpha
 * (what ConvectionFlux::max_eigenvalue computes before :241 overrides it) */
static double lf_eig(double gm, const double* w, int dir) {
    double qn = w[2 + dir];
    double c = sqrt(gm * w[1] / w[0]);
    return dmax(fabs(qn - c), fabs(qn + c));
}

/* One sweep direction: Weno5::x/y/z_sweep (weno-5.cpp:75-220) or
 * Weno5cw::x/y/z_sweep + compute_num_flux (weno-5cw.cpp:4-262).
 * f(i) is the flux at i+1/2 for i from begin-1 to end-1 (nx+1 faces). */
static void sweep(const ns_params* p, const geom* g, int dir, const double* F, const double* U,
                  const double* W, double* f) {
    const int phys = (p->semantics == NS_SEM_PHYSICAL);
    const int borges = (p->weights == NS_WEIGHTS_BORGES);
    const int charw = (p->convection == NS_CONV_WENO5_CHAR);
    const int di = (dir == 0), dj = (dir == 1), dk = (dir == 2);
    const int ib = NG - di, jb = NG - dj, kb = NG - dk;
    double n[3] = {(double)di, (double)dj, (double)dk}, l[3], m[3];
    orthogonal_unit_vectors(n, l, m);
#pragma omp parallel for schedule(static)
    for (int i = ib; i < g->nx + NG; i++)
        for (int j = jb; j < g->ny + NG; j++)
            for (int k = kb; k < g->nz + NG; k++) {
                /* max eigenvalue in the stencil: constant 3.0 (convection_flux.cpp:241) */
                double alpha = 3.0;
                if (phys) {
                    alpha = 0.0;
                    for (int s = -2; s <= 3; s++)
                        alpha = dmax(alpha, lf_eig(p->gamma, W + IX(g, i + s * di, j + s * dj, k + s * dk, 0), dir));
                }
                double fL[5][5], fR[5][5]; /* [q][stencil] */
                for (int s = 0; s < 5; s++) {
                    size_t a = IX(g, i + (s - 2) * di, j + (s - 2) * dj, k + (s - 2) * dk, 0);
                    size_t b = IX(g, i + (s - 1) * di, j + (s - 1) * dj, k + (s - 1) * dk, 0);
                    for (int q = 0; q < 5; q++) {
                        fL[q][s] = (F[a + q] + alpha * U[a + q]) * 0.5;
                        fR[q][s] = (F[b + q] - alpha * U[b + q]) * 0.5;
                    }
                }
                double* out = f + IX(g, i, j, k, 0);
                if (!charw) {
                    for (int q = 0; q < 5; q++) {
                        double fl = weno_left(borges, fL[q][0], fL[q][1], fL[q][2], fL[q][3], fL[q][4]);
                        double fr = weno_right(borges, fR[q][0], fR[q][1], fR[q][2], fR[q][3], fR[q][4]);
                        out[q] = fl + fr;
                    }
                } else {
                    const double* w0 = W + IX(g, i, j, k, 0);
                    const double* w1 = W + IX(g, i + di, j + dj, k + dk, 0);
                    double wa[5];
                    for (int q = 0; q < 5; q++) wa[q] = 0.5 * (w0[q] + w1[q]);
                    double L[5][5], R[5][5];
                    eigenvectors(phys, wa[0], wa[1], wa[2], wa[3], wa[4], p->gamma, n, l, m, L, R);
                    double cL[5][5], cR[5][5], ft[5];
                    /* matrix::square_matrix_matrix_product, src/matrix.cpp:12-20 */
                    for (int r = 0; r < 5; r++)
                        for (int s = 0; s < 5; s++) {
                            cL[r][s] = 0.0; cR[r][s] = 0.0;
                            for (int q = 0; q < 5; q++) {
                                cL[r][s] += L[r][q] * fL[q][s];
                                cR[r][s] += L[r][q] * fR[q][s];
                            }
                        }
                    for (int r = 0; r < 5; r++) {
                        double fl = weno_left(borges, cL[r][0], cL[r][1], cL[r][2], cL[r][3], cL[r][4]);
                        double fr = weno_right(borges, cR[r][0], cR[r][1], cR[r][2], cR[r][3], cR[r][4]);
                        ft[r] = fl + fr;
                    }
                    /* matrix::square_matrix_vector_product, src/matrix.cpp:4-10 */
                    for (int q = 0; q < 5; q++) {
                        out[q] = 0.0;
                        for (int r = 0; r < 5; r++) out[q] += R[q][r] * ft[r];
                    }
                }
            }
}

/* Weno5::solve + compute_residual, weno-5.cpp:3-73: R += (f(i)-f(i-1))/d per axis */
static void convection_solve(const ns_params* p, const geom* g, const double* W,
                             const double* U, double* R) {
    if (p->convection == NS_CONV_NONE) return;
    double* fx = zeros(g);
    double* fy = zeros(g);
    double* fz = zeros(g);
    double* F = zeros(g);
    double* f3[3] = {fx, fy, fz};
    int ndir = (p->dim == 3) ? 3 : 2;
    for (int d = 0; d < ndir; d++) {
        double n[3] = {(double)(d == 0), (double)(d == 1), (double)(d == 2)};
        form_flux(p, g, W, n, F);
        sweep(p, g, d, F, U, W, f3[d]);
    }
    const double dx = g->dx, dy = g->dy, dz = g->dz;
#pragma omp parallel for schedule(static)
    for (int i = NG; i < g->nx + NG; i++)
        for (int j = NG; j < g->ny + NG; j++)
            for (int k = NG; k < g->nz + NG; k++)
                for (int q = 0; q < NQ; q++) {
                    size_t c = IX(g, i, j, k, q);
                    R[c] += (fx[c] - fx[IX(g, i - 1, j, k, q)]) / dx;
                    R[c] += (fy[c] - fy[IX(g, i, j - 1, k, q)]) / dy;
                    R[c] += (fz[c] - fz[IX(g, i, j, k - 1, q)]) / dz;
                }
    free(fx); free(fy); free(fz); free(F);
}

/* ------------------------------------------------------------------------ */
/* Centered differences: src/difference_operators/cd-n.cpp:91-164,
 * coefficients src/difference_operators/cd_constants.hpp:10-28 */

static const double cd2_df[3] = {-1. / 2, 0., 1. / 2.};
static const double cd2_ddf[3] = {1., -2., 1.};
static const double cd4_df[5] = {1. / 12., -2. / 3., 0., 2. / 3., -1. / 12.};
static const double cd4_ddf[5] = {-1. / 12., 4. / 3., -5. / 2., 4. / 3., -1. / 12.};
static const double cd6_df[7] = {-1. / 60., 3. / 20., -3. / 4., 0., 3. / 4., -3. / 20., 1. / 60.};
static const double cd6_ddf[7] = {1. / 90., -3. / 20., 3. / 2., -49. / 18., 3. / 2., -3. / 20., 1. / 90.};

static void cd_coeffs(int order, const double** df, const double** ddf, int* w) {
    if (order == 4) { *df = cd4_df; *ddf = cd4_ddf; *w = 5; }
    else if (order == 6) { *df = cd6_df; *ddf = cd6_ddf; *w = 7; }
    else { *df = cd2_df; *ddf = cd2_ddf; *w = 3; }
}

/* generic_fd_{x,y,z}: df = sum f(.. + start + idx ..) * c[idx] / d over interior
 * (x planes ilo..ihi-1) */
static void generic_fd_range(const geom* g, int ax, const double* f, double* df, const double* c,
                             int w, double d, int ilo, int ihi) {
    const int start = -(w / 2);
#pragma omp parallel for schedule(static)
    for (int i = ilo; i < ihi; i++)
        for (int j = NG; j < g->ny + NG; j++)
            for (int k = NG; k < g->nz + NG; k++)
                for (int q = 0; q < NQ; q++) {
                    double sum = 0.;
                    for (int s = 0; s < w; s++) {
                        int o = start + s;
                        size_t a = IX(g, i + (ax == 0) * o, j + (ax == 1) * o, k + (ax == 2) * o, q);
                        sum += f[a] * c[s] / d;
                    }
                    df[IX(g, i, j, k, q)] = sum;
                }
}

static void generic_fd(const geom* g, int ax, const double* f, double* df, const double* c,
                       int w, double d) {
    generic_fd_range(g, ax, f, df, c, w, d, NG, g->nx + NG);
}

/* DiffusionScheme stress helpers, src/diffusion_schemes/diffusion_scheme.cpp:3-58 */
static double tauxx(double mu, double du_dx, double dv_dy, double lamb) {
    return 2.0 * mu * du_dx + lamb * (du_dx + dv_dy);
}
static double tauyy(double mu, double du_dx, double dv_dy, double lamb) {
    return 2.0 * mu * dv_dy + lamb * (du_dx + dv_dy);
}
static double tauxy(double mu, double du_dy, double dv_dx) { return mu * (du_dy + dv_dx); }
static double dtauxx_dx(double mu, double dmu_dx, double du_dx, double dv_dy, double du_dxdx,
                        double dv_dydx, double lamb, double dlamb_dx) {
    double ret = 2.0 * dmu_dx * du_dx + 2.0 * mu * du_dxdx + dlamb_dx * (du_dx + dv_dy);
    ret += lamb * (du_dxdx + dv_dydx);
    return ret;
}
static double dtauyy_dy(double mu, double dmu_dy, double dv_dy, double dv_dydy, double du_dx,
                        double du_dxdy, double lamb, double dlamb_dy) {
    double ret = 2.0 * dmu_dy * dv_dy + 2.0 * mu * dv_dydy + dlamb_dy * (du_dx + dv_dy);
    ret += lamb * (du_dxdy + dv_dydy);
    return ret;
}
static double dtauxy_dx(double mu, double dmu_dx, double du_dy, double dv_dx, double du_dydx,
                        double dv_dxdx) {
    return dmu_dx * (du_dy + dv_dx) + mu * (du_dydx + dv_dxdx);
}
static double dtauyx_dy(double mu, double dmu_dy, double du_dy, double dv_dx, double du_dydy,
                        double dv_dxdy) {
    return dmu_dy * (du_dy + dv_dx) + mu * (du_dydy + dv_dxdy);
}

enum { Irho = 0, Ip = 1, Iu = 2, Iv = 3, Iw = 4 };

/* CenteredDiffusion::solve + compute_residual, centered_diffusion.cpp:3-182 */
static void diffusion_solve_reference(const ns_params* p, const geom* g, const double* W, double* R) {
    const double *df, *ddf;
    int w;
    cd_coeffs(p->diffusion_order, &df, &ddf, &w);
    double* Dxx = zeros(g);
    double* Dyy = zeros(g);
    double* Dx = zeros(g);
    double* Dy = zeros(g);
    double* Dxy = zeros(g);
    double* Dyx = zeros(g);
    generic_fd(g, 0, W, Dxx, ddf, w, g->dx * g->dx);
    generic_fd(g, 0, W, Dyy, ddf, w, g->dy * g->dy); /* ddf_dydy differentiates along x (cd-n.cpp:77) */
    generic_fd(g, 0, W, Dx, df, w, g->dx);
    /* a slab forms dW/dy on its exchanged x ghost planes too: the neighbour's values,
     * which the reference's communicate(dW_y) brings in across ranks */
    generic_fd_range(g, 1, W, Dy, df, w, g->dy, g->xlo, g->xhi);
    communicate(p, g, Dx); /* centered_diffusion.cpp:22-24: only periodic halos are filled */
    communicate(p, g, Dy);
    generic_fd(g, 1, Dx, Dxy, df, w, g->dy);
    generic_fd(g, 0, Dy, Dyx, df, w, g->dx);
    const double gm = p->gamma, Pr = p->Pr, mu0 = p->mu;
#pragma omp parallel for schedule(static)
    for (int i = NG; i < g->nx + NG; i++)
        for (int j = NG; j < g->ny + NG; j++)
            for (int k = NG; k < g->nz + NG; k++) {
                size_t c = IX(g, i, j, k, 0);
                double mu = mu0, dmu_dx = 0.0, dmu_dy = 0.0;
                double lamb = (-2. / 3.) * mu;
                double dlamb_dx = -(2. / 3.) * dmu_dx;
                double dlamb_dy = -(2. / 3.) * dmu_dy;
                double U = W[c + Iu], V = W[c + Iv], P = W[c + Ip], RHO = W[c + Irho];
                double du_dx = Dx[c + Iu], du_dy = Dy[c + Iu];
                double du_dxdx = Dxx[c + Iu], du_dydy = Dyy[c + Iu];
                double du_dxdy = Dxy[c + Iu], du_dydx = Dyx[c + Iu];
                double dv_dy = Dy[c + Iv], dv_dx = Dx[c + Iv];
                double dv_dxdx = Dxx[c + Iv], dv_dydy = Dyy[c + Iv];
                double dv_dydx = Dyx[c + Iv], dv_dxdy = Dxy[c + Iv];
                double drho_dx = Dx[c + Irho], dp_dx = Dx[c + Ip];
                double drho_dxdx = Dxx[c + Irho], dp_dxdx = Dxx[c + Ip];
                double drho_dy = Dy[c + Irho], dp_dy = Dy[c + Ip];
                double drho_dydy = Dyy[c + Irho], dp_dydy = Dyy[c + Ip];
                double Dtauxx_dx = dtauxx_dx(mu, dmu_dx, du_dx, dv_dy, du_dxdx, dv_dydx, lamb, dlamb_dx);
                double Dtauyy_dy = dtauyy_dy(mu, dmu_dy, dv_dy, dv_dydy, du_dx, du_dxdy, lamb, dlamb_dy);
                double Dtauxy_dx = dtauxy_dx(mu, dmu_dx, du_dy, dv_dx, du_dydx, dv_dxdx);
                double Dtauyx_dy = dtauyx_dy(mu, dmu_dy, du_dy, dv_dx, du_dydy, dv_dxdy);
                double Tauxx = tauxx(mu, du_dx, dv_dy, lamb);
                double Tauyy = tauxx(mu, du_dx, dv_dy, lamb); /* :143 uses tauxx */
                double Tauxy = tauxy(mu, du_dy, dv_dx);
                double Tauyx = Tauxy;
                double Dtauvx_dx = U * Dtauxx_dx + V * Dtauxy_dx + Tauxx * du_dx + Tauxy * dv_dy; /* :148 */
                double Dtauvy_dy = U * Dtauyx_dy + V * Dtauyy_dy + Tauyy * dv_dy + Tauyx * du_dy;
                double one_rho = 1. / RHO;
                double one_rho2 = 1. / (RHO * RHO);
                double one_rho3 = 1. / (RHO * RHO * RHO);
                double temp1 = dmu_dx * (one_rho * dp_dx - P * one_rho2 * drho_dx);
                double temp2 = mu * (2.0 * one_rho2 * drho_dx * dp_dx + one_rho * dp_dxdx +
                                     one_rho3 * P * drho_dx * drho_dx - one_rho2 * P * drho_dxdx);
                double temp3 = gm / (Pr * (gm - 1.0));
                double Dqx_dx = -temp3 * (temp1 + temp2);
                temp1 = dmu_dy * (one_rho * dp_dy - P * one_rho2 * drho_dy);
                /* :166 multiplies by the enum index p (= 1) instead of the pressure */
                temp2 = mu * (2.0 * one_rho2 * drho_dy * dp_dy + one_rho * dp_dydy +
                              one_rho3 * (double)Ip * drho_dy * drho_dy - one_rho2 * P * drho_dydy);
                double Dqy_dy = -temp3 * (temp1 + temp2);
                double x_mom = -Dtauxx_dx - Dtauyx_dy;
                double y_mom = -Dtauyy_dy - Dtauxy_dx;
                double ene = -Dtauvx_dx - Dtauvy_dy + Dqx_dx + Dqy_dy;
                R[c + Ip] += ene;
                R[c + Iu] += x_mom;
                R[c + Iv] += y_mom;
                R[c + Iw] -= 0.0;
            }
    free(Dxx); free(Dyy); free(Dx); free(Dy); free(Dxy); free(Dyx);
}

/* Physical semantics (no reference counterpart): full 3D compressible viscous
 * and heat-flux terms with constant mu, Stokes lambda = -2/3 mu, central
 * differences of the chosen order, mixed derivatives as tensor-product
 * stencils over the boundary-filled primitive field. */
static double pick(const double* A, const geom* g, int i, int j, int k, int q) {
    return A[IX(g, i, j, k, q)];
}

static void diffusion_solve_physical(const ns_params* p, const geom* g, const double* W, double* R) {
    const double *df, *ddf;
    int w;
    cd_coeffs(p->diffusion_order, &df, &ddf, &w);
    const int h = w / 2;
    const double d[3] = {g->dx, g->dy, g->dz};
    const int nd = (p->dim == 3) ? 3 : 2;
    const double gm = p->gamma, mu = p->mu, lamb = (-2. / 3.) * p->mu;
    const double kap = gm / (p->Pr * (gm - 1.0)) * mu; /* k/cv-scaled heat conductivity on p/rho */
    /* neighbours of a corner/edge halo cell: clamp into the filled region */
#pragma omp parallel for schedule(static)
    for (int i = NG; i < g->nx + NG; i++)
        for (int j = NG; j < g->ny + NG; j++)
            for (int k = NG; k < g->nz + NG; k++) {
                int c3[3] = {i, j, k};
                double gu[3][3], lap[3], gdiv[3], gT[3], lapT = 0.0;
                /* first derivatives of u,v,w and T = p/rho; second derivatives */
                for (int a = 0; a < 3; a++) {
                    lap[a] = 0.0;
                    for (int b = 0; b < 3; b++) gu[a][b] = 0.0;
                    gdiv[a] = 0.0;
                    gT[a] = 0.0;
                }
                for (int b = 0; b < nd; b++) {
                    for (int s = 0; s < w; s++) {
                        int o = s - h;
                        int ii = i + (b == 0) * o, jj = j + (b == 1) * o, kk = k + (b == 2) * o;
                        double T = pick(W, g, ii, jj, kk, Ip) / pick(W, g, ii, jj, kk, Irho);
                        for (int a = 0; a < 3; a++) {
                            double va = pick(W, g, ii, jj, kk, Iu + a);
                            gu[a][b] += va * (df[s] / d[b]);
                            lap[a] += va * (ddf[s] / (d[b] * d[b]));
                        }
                        gT[b] += T * (df[s] / d[b]);
                        lapT += T * (ddf[s] / (d[b] * d[b]));
                    }
                }
                /* grad(div u)_a = sum_b d2 u_b / dx_a dx_b */
                for (int a = 0; a < nd; a++)
                    for (int b = 0; b < nd; b++) {
                        double acc = 0.0;
                        if (a == b) {
                            for (int s = 0; s < w; s++) {
                                int o = s - h;
                                int ii = i + (a == 0) * o, jj = j + (a == 1) * o, kk = k + (a == 2) * o;
                                acc += pick(W, g, ii, jj, kk, Iu + b) * (ddf[s] / (d[a] * d[a]));
                            }
                        } else {
                            for (int s = 0; s < w; s++)
                                for (int t = 0; t < w; t++) {
                                    int o1 = s - h, o2 = t - h;
                                    int ii = i + (a == 0) * o1 + (b == 0) * o2;
                                    int jj = j + (a == 1) * o1 + (b == 1) * o2;
                                    int kk = k + (a == 2) * o1 + (b == 2) * o2;
                                    /* corner halos are not filled by the boundary fill: fold them back */
                                    int cc[3] = {ii, jj, kk};
                                    const int nn[3] = {g->nx, g->ny, g->nz};
                                    for (int e = 0; e < 3; e++) {
                                        if (e == 0 && g->ext) continue; /* ghost planes: the neighbours' cells */
                                        if (cc[e] < NG || cc[e] >= nn[e] + NG) {
                                            if (p->bc[e] == NS_BC_PERIODIC)
                                                cc[e] = NG + ((cc[e] - NG) % nn[e] + nn[e]) % nn[e];
                                            else
                                                cc[e] = cc[e] < NG ? NG : nn[e] + NG - 1;
                                        }
                                    }
                                    acc += pick(W, g, cc[0], cc[1], cc[2], Iu + b) *
                                           (df[s] / d[a]) * (df[t] / d[b]);
                                }
                        }
                        gdiv[a] += acc;
                    }
                (void)c3;
                size_t c = IX(g, i, j, k, 0);
                double uv[3] = {W[c + Iu], W[c + Iv], W[c + Iw]};
                double div = 0.0;
                for (int a = 0; a < 3; a++) div += gu[a][a];
                double mom[3], work = 0.0, diss = 0.0;
                for (int a = 0; a < 3; a++) {
                    /* d tau_ab / dx_b = mu lap u_a + (mu + lamb) d(div u)/dx_a */
                    mom[a] = mu * lap[a] + (mu + lamb) * gdiv[a];
                    work += uv[a] * mom[a];
                }
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        double tab = mu * (gu[a][b] + gu[b][a]) + (a == b ? lamb * div : 0.0);
                        diss += tab * gu[a][b];
                    }
                R[c + Iu] -= mom[0];
                R[c + Iv] -= mom[1];
                R[c + Iw] -= mom[2];
                R[c + Ip] -= work + diss + kap * lapT;
            }
}

static void diffusion_solve(const ns_params* p, const geom* g, const double* W, double* R) {
    if (p->diffusion == NS_DIFF_NONE) return;
    if (p->semantics == NS_SEM_PHYSICAL)
        diffusion_solve_physical(p, g, W, R);
    else
        diffusion_solve_reference(p, g, W, R);
}

/* ------------------------------------------------------------------------ */
/* Time step: src/time_scheme.cpp:3-136, src/eq_of_state.cpp:89-101 */

static double local_max_dt(const ns_params* p, const geom* g, const double* W) {
    double best = 1E10;
    const double gm = p->gamma, dx = g->dx, dy = g->dy, dz = g->dz;
    const int phys = (p->semantics == NS_SEM_PHYSICAL);
    for (int i = NG; i < g->nx + NG; i++)
        for (int j = NG; j < g->ny + NG; j++)
            for (int k = NG; k < g->nz + NG; k++) {
                const double* w = W + IX(g, i, j, k, 0);
                double rho = w[0], pr = w[1], u = w[2], v = w[3], ww = w[4];
                double c = sqrt(gm * pr / rho);
                double ex = dx / dmax(fabs(u + c), fabs(u - c));
                double ey = dy / dmax(fabs(v + c), fabs(v - c));
                double ez = dz / dmax(fabs(ww + c), fabs(ww - c));
                double dt;
                if (phys) {
                    /* sum of the directional rates: the stable multi-dimensional CFL */
                    double rate = 1.0 / ex + 1.0 / ey + ((p->dim == 3) ? 1.0 / ez : 0.0);
                    dt = 1.0 / rate;
                } else {
                    dt = dmin(dmin(ex, ey), ez);
                }
                if (dt < best) best = dt;
            }
    return best;
}

static void substep(const geom* g, double* now, const double* prev, const double* inc, double m1,
                    double m2, double m3) {
#pragma omp parallel for schedule(static)
    for (int i = NG; i < g->nx + NG; i++)
        for (int j = NG; j < g->ny + NG; j++)
            for (int k = NG; k < g->nz + NG; k++)
                for (int q = 0; q < NQ; q++) {
                    size_t c = IX(g, i, j, k, q);
                    now[c] = (prev[c] * m1) + (now[c] * m2) + (inc[c] * m3);
                }
}

static void interior_copy(const geom* g, const double* in, double* out) {
    for (int i = NG; i < g->nx + NG; i++)
        for (int j = NG; j < g->ny + NG; j++)
            for (int k = NG; k < g->nz + NG; k++)
                for (int q = 0; q < NQ; q++) out[IX(g, i, j, k, q)] = in[IX(g, i, j, k, q)];
}

static int check(const ns_params* p) {
    if (!p || p->nx < 1 || p->ny < 1 || p->nz < 1) return 1;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* exported entry points (all arrays halo'd AoS) */

size_t nso_array_elems(const ns_params* p) {
    geom g = make_geom(p);
    return n_all(&g);
}

int nso_convection_solve(const ns_params* p, const double* W, const double* U, double* R) {
    if (check(p)) return 1;
    geom g = make_geom(p);
    convection_solve(p, &g, W, U, R);
    return 0;
}

int nso_diffusion_solve(const ns_params* p, const double* W, double* R) {
    if (check(p)) return 1;
    geom g = make_geom(p);
    diffusion_solve(p, &g, W, R);
    return 0;
}

/* one sweep's face flux array (f(i) at i+1/2, reference indexing) */
int nso_face_flux(const ns_params* p, int dir, const double* W, const double* U, double* f) {
    if (check(p) || dir < 0 || dir > 2) return 1;
    geom g = make_geom(p);
    double* F = zeros(&g);
    double n[3] = {(double)(dir == 0), (double)(dir == 1), (double)(dir == 2)};
    form_flux(p, &g, W, n, F);
    sweep(p, &g, dir, F, U, W, f);
    free(F);
    return 0;
}

/* stage prologue of time_scheme.cpp:124,133-135 applied to a primitive field:
 * U = cons(W) on all cells, boundary fill + exchange of U, W = prim(U) */
int nso_prologue(const ns_params* p, double* W, double* U) {
    if (check(p)) return 1;
    geom g = make_geom(p);
    prim_to_cons(p, &g, W, U);
    neumann_fill(p, &g, U);
    communicate(p, &g, U);
    cons_to_prim(p, &g, U, W);
    return 0;
}

int nso_rhs(const ns_params* p, const double* Win, double* R, int terms) {
    if (check(p)) return 1;
    geom g = make_geom(p);
    double* W = (double*)malloc(n_all(&g) * sizeof(double));
    memcpy(W, Win, n_all(&g) * sizeof(double));
    double* U = zeros(&g);
    nso_prologue(p, W, U);
    for (int i = NG; i < g.nx + NG; i++)
        for (int j = NG; j < g.ny + NG; j++)
            for (int k = NG; k < g.nz + NG; k++)
                for (int q = 0; q < NQ; q++) R[IX(&g, i, j, k, q)] = 0.0;
    if (terms & NS_TERM_CONVECTION) convection_solve(p, &g, W, U, R);
    if (terms & NS_TERM_DIFFUSION) diffusion_solve(p, &g, W, R);
    free(W); free(U);
    return 0;
}

int nso_compute_dt(const ns_params* p, const double* W, double* dt) {
    if (check(p)) return 1;
    geom g = make_geom(p);
    *dt = local_max_dt(p, &g, W) * p->cfl;
    return 0;
}

/* TimeScheme::step, time_scheme.cpp:3-70.  W in/out, U out (both halo'd). */
int nso_time_step(const ns_params* p, double* W, double* U, double* dt_out) {
    if (check(p)) return 1;
    geom g = make_geom(p);
    double* R = zeros(&g);
    double* Uprev = zeros(&g);
    double dt = local_max_dt(p, &g, W) * p->cfl;
    prim_to_cons(p, &g, W, U);
    interior_copy(&g, U, Uprev);
    const double m1s[3] = {1.0, 3.0 / 4.0, 1. / 3.};
    const double m2s[3] = {0.0, 1.0 / 4.0, 2. / 3.};
    const double m3s[3] = {-dt, -(1. / 4.) * dt, -(2. / 3.) * dt};
    for (int s = 0; s < 3; s++) {
        memset(R, 0, n_all(&g) * sizeof(double));
        neumann_fill(p, &g, U);
        communicate(p, &g, U);
        cons_to_prim(p, &g, U, W);
        convection_solve(p, &g, W, U, R);
        diffusion_solve(p, &g, W, R);
        substep(&g, U, Uprev, R, m1s[s], m2s[s], m3s[s]);
    }
    cons_to_prim(p, &g, U, W);
    if (dt_out) *dt_out = dt;
    free(R); free(Uprev);
    return 0;
}

/* Slab decomposition along x (bc[0] = NS_BC_EXTERNAL): nsteps of TimeScheme::step
 * on one slab, with the halo exchange and dt reduction of the reference's MPI
 * path (communicator.cpp:16-57, time_scheme.cpp:127-136) delegated to fn:
 *   fn(user, 0, &dt_min): replace the slab's CFL minimum by the minimum over slabs
 *   fn(user, 1, U): fill U's x ghost planes (interior j, k) from the neighbours
 * fn returns 0 on success. */
typedef int (*nso_exchange_fn)(void* user, int what, double* data);

int nso_slab_run(const ns_params* p, double* W, double* U, int nsteps, double* dts, nso_exchange_fn fn,
                 void* user) {
    if (check(p) || !fn) return 1;
    geom g = make_geom(p);
    double* R = zeros(&g);
    double* Uprev = zeros(&g);
    const double m1s[3] = {1.0, 3.0 / 4.0, 1. / 3.};
    const double m2s[3] = {0.0, 1.0 / 4.0, 2. / 3.};
    int rc = 0;
    for (int s = 0; s < nsteps && !rc; s++) {
        double m = local_max_dt(p, &g, W);
        if (fn(user, 0, &m)) { rc = 2; break; }
        double dt = m * p->cfl;
        const double m3s[3] = {-dt, -(1. / 4.) * dt, -(2. / 3.) * dt};
        prim_to_cons(p, &g, W, U);
        interior_copy(&g, U, Uprev);
        for (int st = 0; st < 3; st++) {
            memset(R, 0, n_all(&g) * sizeof(double));
            if (fn(user, 1, U)) { rc = 2; break; }
            neumann_fill(p, &g, U);
            communicate(p, &g, U);
            cons_to_prim(p, &g, U, W);
            convection_solve(p, &g, W, U, R);
            diffusion_solve(p, &g, W, R);
            substep(&g, U, Uprev, R, m1s[st], m2s[st], m3s[st]);
        }
        if (rc) break;
        cons_to_prim(p, &g, U, W);
        if (dts) dts[s] = dt;
    }
    free(R); free(Uprev);
    return rc;
}

/* n steps; dts (may be NULL) receives each step's dt */
int nso_run(const ns_params* p, double* W, double* U, int nsteps, double* dts) {
    for (int s = 0; s < nsteps; s++) {
        double dt;
        int rc = nso_time_step(p, W, U, &dt);
        if (rc) return rc;
        if (dts) dts[s] = dt;
    }
    return 0;
}
