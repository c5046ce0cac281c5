/*
 * mf3d_oracle.c -- CPU restatement of MacroFlow3D's Darcy head-solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product in
 * macroflow3d_b200/csrc: it is loaded by tests/, by __graft_entry__.smoke() and
 * by bench.py's CPU-baseline leg, never by the product path.
 *
 * Every function restates one reference routine with the same arithmetic
 * (same harmonic-mean form, same accumulation order, same boundary and pin
 * conventions) so that oracle and reference agree to rounding.  Citations are
 * to files of santi-esquerre/MacroFlow3D.
 *
 * Parity pin: the reference has no golden vectors for this path; the oracle is
 * pinned against outputs of the reference's own CUDA code, compiled from its
 * sources by oracle/Makefile into oracle/_ref and run on a B200
 * (tests/golden/make_golden.py writes the fixtures, tests/test_oracle_golden.py
 * checks them).
 *
 * Layout: cell (i,j,k) lives at i + nx*(j + ny*k) (src/core/Grid3D.hpp:54).
 * BC types follow src/core/BCSpec.hpp:13 (0 Dirichlet, 1 Neumann, 2 Periodic),
 * face order xmin,xmax,ymin,ymax,zmin,zmax (src/core/BCSpecDevice.cuh:26-47).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { OG_DIRICHLET = 0, OG_NEUMANN = 1, OG_PERIODIC = 2 };

typedef struct {
    int type[6];
    double value[6];
} og_bc;

#define IX(i, j, k) ((size_t)(i) + (size_t)nx * ((size_t)(j) + (size_t)ny * (size_t)(k)))

static inline double hmean(double a, double b) { return 2.0 / (1.0 / a + 1.0 / b); }

int og_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void og_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------ */
/* Neighbour value + coefficient in one direction.                           */
/* src/multigrid/smoothers/bc_stencil_helpers.cuh:33-271                      */
/* dir: 0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+                                    */
/* ------------------------------------------------------------------------ */
static inline void og_neighbor(int nx, int ny, int nz, const og_bc* bc, const double* x,
                               const double* K, int i, int j, int k, int dir, double* val,
                               double* coef) {
    const size_t c = IX(i, j, k);
    const double Kc = K[c];
    int ni = i, nj = j, nk = k, at_bnd = 0;
    switch (dir) {
    case 0: at_bnd = (i == 0); ni = at_bnd ? nx - 1 : i - 1; break;
    case 1: at_bnd = (i == nx - 1); ni = at_bnd ? 0 : i + 1; break;
    case 2: at_bnd = (j == 0); nj = at_bnd ? ny - 1 : j - 1; break;
    case 3: at_bnd = (j == ny - 1); nj = at_bnd ? 0 : j + 1; break;
    case 4: at_bnd = (k == 0); nk = at_bnd ? nz - 1 : k - 1; break;
    default: at_bnd = (k == nz - 1); nk = at_bnd ? 0 : k + 1; break;
    }
    if (!at_bnd || bc->type[dir] == OG_PERIODIC) {
        const size_t n = IX(ni, nj, nk);
        *val = x[n];
        *coef = hmean(Kc, K[n]);
    } else if (bc->type[dir] == OG_NEUMANN) {
        *val = x[c];
        *coef = 0.0;
    } else { /* Dirichlet: ghost contributes only to the diagonal */
        *val = 0.0;
        *coef = 2.0 * Kc;
    }
}

static inline int og_is_interior(int nx, int ny, int nz, int i, int j, int k) {
    return i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2;
}

/* ------------------------------------------------------------------------ */
/* y = A x  (negative definite).  src/numerics/operators/varcoeff_laplacian.cu */
/* interior :38-73, boundary :80-239 (pin adds only in-domain coefficients).  */
/* ------------------------------------------------------------------------ */
void og_apply_A(int nx, int ny, int nz, double dx, const og_bc* bc, int pin, const double* K,
                const double* x, double* y) {
    const double inv_dx2 = 1.0 / (dx * dx);
    const int stride = nx * ny;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t idx = IX(i, j, k);
                const double xC = x[idx], KC = K[idx];
                if (og_is_interior(nx, ny, nz, i, j, k)) {
                    const double Kxm = hmean(KC, K[idx - 1]);
                    const double Kxp = hmean(KC, K[idx + 1]);
                    const double Kym = hmean(KC, K[idx - nx]);
                    const double Kyp = hmean(KC, K[idx + nx]);
                    const double Kzm = hmean(KC, K[idx - stride]);
                    const double Kzp = hmean(KC, K[idx + stride]);
                    const double Ax = Kxm * (xC - x[idx - 1]) + Kxp * (xC - x[idx + 1]) +
                                      Kym * (xC - x[idx - nx]) + Kyp * (xC - x[idx + nx]) +
                                      Kzm * (xC - x[idx - stride]) + Kzp * (xC - x[idx + stride]);
                    y[idx] = -Ax * inv_dx2;
                    continue;
                }
                double Ax = 0.0, aC = 0.0;
                /* six directions in the reference's order x-, x+, y-, y+, z-, z+ */
                for (int d = 0; d < 6; ++d) {
                    int at_bnd, ni = i, nj = j, nk = k;
                    switch (d) {
                    case 0: at_bnd = (i == 0); ni = at_bnd ? nx - 1 : i - 1; break;
                    case 1: at_bnd = (i == nx - 1); ni = at_bnd ? 0 : i + 1; break;
                    case 2: at_bnd = (j == 0); nj = at_bnd ? ny - 1 : j - 1; break;
                    case 3: at_bnd = (j == ny - 1); nj = at_bnd ? 0 : j + 1; break;
                    case 4: at_bnd = (k == 0); nk = at_bnd ? nz - 1 : k - 1; break;
                    default: at_bnd = (k == nz - 1); nk = at_bnd ? 0 : k + 1; break;
                    }
                    if (!at_bnd) {
                        const size_t n = IX(ni, nj, nk);
                        const double Kh = hmean(KC, K[n]);
                        Ax += Kh * (xC - x[n]);
                        aC += Kh;
                    } else if (bc->type[d] == OG_PERIODIC) {
                        const size_t n = IX(ni, nj, nk);
                        const double Kh = hmean(KC, K[n]);
                        Ax += Kh * (xC - x[n]);
                    } else if (bc->type[d] == OG_DIRICHLET) {
                        Ax += 2.0 * KC * xC;
                    }
                }
                if (pin && idx == 0) Ax += aC * xC;
                y[idx] = -Ax * inv_dx2;
            }
}

/* One GSRB cell update.  Interior form: src/multigrid/smoothers/gsrb_3d.cu:29-73;
 * boundary form (faces/edges/vertices): gsrb_3d.cu:76-363. */
static inline double og_gsrb_cell(int nx, int ny, int nz, double dx2, const og_bc* bc, int pin,
                                  const double* K, const double* b, const double* x, int i,
                                  int j, int k) {
    const int stride = nx * ny;
    const size_t idx = IX(i, j, k);
    if (og_is_interior(nx, ny, nz, i, j, k)) {
        const double KC = K[idx];
        const double K_xp = hmean(KC, K[idx + 1]);
        const double K_xm = hmean(KC, K[idx - 1]);
        const double K_yp = hmean(KC, K[idx + nx]);
        const double K_ym = hmean(KC, K[idx - nx]);
        const double K_zp = hmean(KC, K[idx + stride]);
        const double K_zm = hmean(KC, K[idx - stride]);
        double result = x[idx + 1] * K_xp;
        result += x[idx - 1] * K_xm;
        result += x[idx + nx] * K_yp;
        result += x[idx - nx] * K_ym;
        result += x[idx + stride] * K_zp;
        result += x[idx - stride] * K_zm;
        const double aC = K_xp + K_xm + K_yp + K_ym + K_zp + K_zm;
        return (result - b[idx] * dx2) / aC;
    }
    double v[6], c[6];
    for (int d = 0; d < 6; ++d) og_neighbor(nx, ny, nz, bc, x, K, i, j, k, d, &v[d], &c[d]);
    const double result = c[0] * v[0] + c[1] * v[1] + c[2] * v[2] + c[3] * v[3] + c[4] * v[4] +
                          c[5] * v[5];
    double aC = c[0] + c[1] + c[2] + c[3] + c[4] + c[5];
    const double b_adj = b[idx] + 0.0;
    if (pin && i == 0 && j == 0 && k == 0) aC *= 2.0;
    return (result - b_adj * dx2) / aC;
}

/* gsrb_smooth_3d: src/multigrid/smoothers/gsrb_3d.cu:368-576.  Red = (i+j+k) even,
 * then black; each colour reads only the other colour, so in-place is exact. */
void og_gsrb(int nx, int ny, int nz, double dx, const og_bc* bc, int pin, const double* K,
             const double* b, double* x, int iters) {
    const double dx2 = dx * dx;
    for (int it = 0; it < iters; ++it)
        for (int color = 0; color < 2; ++color) {
#pragma omp parallel for schedule(static)
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < ny; ++j) {
                    int i0 = (color + j + k) & 1;
                    for (int i = i0; i < nx; i += 2)
                        x[IX(i, j, k)] = og_gsrb_cell(nx, ny, nz, dx2, bc, pin, K, b, x, i, j, k);
                }
        }
}

/* r = b - A x.  Interior: src/multigrid/smoothers/residual_3d.cu:30-80;
 * boundary: residual_3d.cu:83-376 (pin adds the full diagonal at cell 0). */
void og_residual(int nx, int ny, int nz, double dx, const og_bc* bc, int pin, const double* K,
                 const double* x, const double* b, double* r) {
    const double inv_dx2 = 1.0 / (dx * dx);
    const double dx2 = dx * dx;
    const int stride = nx * ny;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t idx = IX(i, j, k);
                if (og_is_interior(nx, ny, nz, i, j, k)) {
                    const double xc = x[idx], Kc = K[idx];
                    double Ax = 0.0;
                    Ax -= 2.0 * (xc - x[idx + 1]) / (1.0 / Kc + 1.0 / K[idx + 1]);
                    Ax -= 2.0 * (xc - x[idx + nx]) / (1.0 / Kc + 1.0 / K[idx + nx]);
                    Ax -= 2.0 * (xc - x[idx - 1]) / (1.0 / Kc + 1.0 / K[idx - 1]);
                    Ax -= 2.0 * (xc - x[idx - nx]) / (1.0 / Kc + 1.0 / K[idx - nx]);
                    Ax -= 2.0 * (xc - x[idx + stride]) / (1.0 / Kc + 1.0 / K[idx + stride]);
                    Ax -= 2.0 * (xc - x[idx - stride]) / (1.0 / Kc + 1.0 / K[idx - stride]);
                    r[idx] = b[idx] - Ax * inv_dx2;
                    continue;
                }
                double v[6], c[6];
                for (int d = 0; d < 6; ++d)
                    og_neighbor(nx, ny, nz, bc, x, K, i, j, k, d, &v[d], &c[d]);
                const double xC = x[idx];
                double result = c[0] * (xC - v[0]) + c[1] * (xC - v[1]) + c[2] * (xC - v[2]) +
                                c[3] * (xC - v[3]) + c[4] * (xC - v[4]) + c[5] * (xC - v[5]);
                if (pin && idx == 0) {
                    const double aC = c[0] + c[1] + c[2] + c[3] + c[4] + c[5];
                    result += aC * xC;
                }
                const double b_adj = b[idx] + 0.0;
                r[idx] = b_adj - (-result / dx2);
            }
}

/* b_c = (1/8) sum of the 8 children.  src/multigrid/transfer/restrict_3d.cu:12-53.
 * NX,NY,NZ are the coarse sizes; the fine grid is exactly twice as large. */
void og_restrict(int NX, int NY, int NZ, const double* rf, double* bc) {
    const int Nx = 2 * NX, Ny = 2 * NY;
    const size_t stride = (size_t)Nx * Ny;
#pragma omp parallel for schedule(static)
    for (int IZ = 0; IZ < NZ; ++IZ)
        for (int IY = 0; IY < NY; ++IY)
            for (int IX_ = 0; IX_ < NX; ++IX_) {
                const size_t in = (size_t)(2 * IX_) + (size_t)(2 * IY) * Nx + (size_t)(2 * IZ) * stride;
                double s = 0.0;
                s += rf[in];
                s += rf[in + 1];
                s += rf[in + Nx];
                s += rf[in + 1 + Nx];
                s += rf[in + stride];
                s += rf[in + 1 + stride];
                s += rf[in + Nx + stride];
                s += rf[in + 1 + Nx + stride];
                bc[(size_t)IX_ + (size_t)IY * NX + (size_t)IZ * NX * NY] = s / 8.0;
            }
}

/* x_f += e_c at the parent cell.  src/multigrid/transfer/prolong_3d.cu:30-621: the
 * octant/offset arithmetic of the 27 kernels reduces to parent (i/2, j/2, k/2). */
void og_prolong_add(int NX, int NY, int NZ, const double* xc, double* xf) {
    const int nx = 2 * NX, ny = 2 * NY, nz = 2 * NZ;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                xf[IX(i, j, k)] += xc[(size_t)(i / 2) + (size_t)NX * ((size_t)(j / 2) + (size_t)NY * (k / 2))];
}

/* Geometric mean of the 8 children.  src/physics/flow/coarsen_K.cu:15-53. */
void og_coarsen_K(int NX, int NY, int NZ, const double* Kf, double* Kc) {
    const int Nx = 2 * NX, Ny = 2 * NY;
    const size_t stride = (size_t)Nx * Ny;
#pragma omp parallel for schedule(static)
    for (int IZ = 0; IZ < NZ; ++IZ)
        for (int IY = 0; IY < NY; ++IY)
            for (int IX_ = 0; IX_ < NX; ++IX_) {
                const size_t i000 = (size_t)(2 * IX_) + (size_t)(2 * IY) * Nx + (size_t)(2 * IZ) * stride;
                const size_t i001 = i000 + stride;
                const double ls = log(Kf[i000]) + log(Kf[i000 + 1]) + log(Kf[i000 + Nx]) +
                                  log(Kf[i000 + 1 + Nx]) + log(Kf[i001]) + log(Kf[i001 + 1]) +
                                  log(Kf[i001 + Nx]) + log(Kf[i001 + 1 + Nx]);
                Kc[(size_t)IX_ + (size_t)IY * NX + (size_t)IZ * NX * NY] = exp(ls / 8.0);
            }
}

/* b = 0; b -= 2 h_bc K_c / dx^2 on every Dirichlet face cell.
 * src/physics/flow/rhs_head.cu:21-194 (faces applied xmin,xmax,ymin,ymax,zmin,zmax). */
void og_build_rhs(int nx, int ny, int nz, double dx, const og_bc* bc, const double* K, double* b) {
    const double inv_dx2 = 1.0 / (dx * dx);
    const size_t n = (size_t)nx * ny * nz;
    memset(b, 0, n * sizeof(double));
    for (int f = 0; f < 6; ++f) {
        if (bc->type[f] != OG_DIRICHLET) continue;
        const double h = bc->value[f];
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    int on = (f == 0 && i == 0) || (f == 1 && i == nx - 1) || (f == 2 && j == 0) ||
                             (f == 3 && j == ny - 1) || (f == 4 && k == 0) || (f == 5 && k == nz - 1);
                    if (!on) continue;
                    const size_t idx = IX(i, j, k);
                    b[idx] -= 2.0 * h * K[idx] * inv_dx2;
                }
    }
}

/* x-linear guess when both x faces are Dirichlet, else zero.
 * src/physics/flow/solve_head.cu:29-73. */
void og_init_guess(int nx, int ny, int nz, const og_bc* bc, double* h) {
    const size_t n = (size_t)nx * ny * nz;
    if (bc->type[0] == OG_DIRICHLET && bc->type[1] == OG_DIRICHLET) {
        const double hw = bc->value[0], he = bc->value[1];
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double t = ((double)i + 0.5) / (double)nx;
                    h[IX(i, j, k)] = hw + (he - hw) * t;
                }
    } else {
        memset(h, 0, n * sizeof(double));
    }
}

/* ------------------------------------------------------------------------ */
/* Multigrid hierarchy and V-cycle                                           */
/* ------------------------------------------------------------------------ */
typedef struct {
    int nl;
    int nx[32], ny[32], nz[32];
    double dx[32];
    double *x[32], *b[32], *r[32], *K[32];
} og_hier;

/* MGHierarchy: halve every axis while num_levels allows, stop when an axis < 2.
 * src/multigrid/mg_types.hpp:86-99. */
static void og_hier_build(og_hier* H, int nx, int ny, int nz, double dx, int num_levels) {
    memset(H, 0, sizeof(*H));
    int cx = nx, cy = ny, cz = nz;
    double cdx = dx;
    for (int l = 0; l < num_levels && l < 32; ++l) {
        const size_t n = (size_t)cx * cy * cz;
        H->nx[l] = cx; H->ny[l] = cy; H->nz[l] = cz; H->dx[l] = cdx;
        H->x[l] = (double*)calloc(n, sizeof(double));
        H->b[l] = (double*)calloc(n, sizeof(double));
        H->r[l] = (double*)calloc(n, sizeof(double));
        H->K[l] = (double*)calloc(n, sizeof(double));
        H->nl = l + 1;
        if (l < num_levels - 1) {
            cx /= 2; cy /= 2; cz /= 2; cdx *= 2.0;
            if (cx < 2 || cy < 2 || cz < 2) break;
        }
    }
}

static void og_hier_free(og_hier* H) {
    for (int l = 0; l < H->nl; ++l) {
        free(H->x[l]); free(H->b[l]); free(H->r[l]); free(H->K[l]);
    }
    H->nl = 0;
}

typedef struct {
    int pre, post, coarse_iters;
} og_mgcfg;

/* v_cycle_recursive: src/multigrid/cycle/v_cycle.cu:36-74. */
static void og_vcycle_rec(og_hier* H, int l, const og_mgcfg* c, const og_bc* bc, int pin) {
    const int nx = H->nx[l], ny = H->ny[l], nz = H->nz[l];
    if (l == H->nl - 1) {
        og_gsrb(nx, ny, nz, H->dx[l], bc, pin, H->K[l], H->b[l], H->x[l], c->coarse_iters);
        return;
    }
    og_gsrb(nx, ny, nz, H->dx[l], bc, pin, H->K[l], H->b[l], H->x[l], c->pre);
    og_residual(nx, ny, nz, H->dx[l], bc, pin, H->K[l], H->x[l], H->b[l], H->r[l]);
    og_restrict(H->nx[l + 1], H->ny[l + 1], H->nz[l + 1], H->r[l], H->b[l + 1]);
    memset(H->x[l + 1], 0, (size_t)H->nx[l + 1] * H->ny[l + 1] * H->nz[l + 1] * sizeof(double));
    og_vcycle_rec(H, l + 1, c, bc, pin);
    og_prolong_add(H->nx[l + 1], H->ny[l + 1], H->nz[l + 1], H->x[l + 1], H->x[l]);
    og_gsrb(nx, ny, nz, H->dx[l], bc, pin, H->K[l], H->b[l], H->x[l], c->post);
}

/* Copy K to level 0 and coarsen to every level: src/physics/flow/solve_head.cu:104-114. */
static void og_hier_set_K(og_hier* H, const double* K) {
    const size_t n0 = (size_t)H->nx[0] * H->ny[0] * H->nz[0];
    memcpy(H->K[0], K, n0 * sizeof(double));
    for (int l = 0; l + 1 < H->nl; ++l)
        og_coarsen_K(H->nx[l + 1], H->ny[l + 1], H->nz[l + 1], H->K[l], H->K[l + 1]);
}

/* MultigridPreconditioner::apply: z = V-cycle(r) from a zero guess.
 * src/numerics/solvers/mg_preconditioner.cu:16-44. */
static void og_mg_apply(og_hier* H, const og_mgcfg* c, const og_bc* bc, int pin, const double* r,
                        double* z) {
    const size_t n0 = (size_t)H->nx[0] * H->ny[0] * H->nz[0];
    memcpy(H->b[0], r, n0 * sizeof(double));
    memset(H->x[0], 0, n0 * sizeof(double));
    og_vcycle_rec(H, 0, c, bc, pin);
    memcpy(z, H->x[0], n0 * sizeof(double));
}

/* Exported V-cycle preconditioner apply (builds its own hierarchy). */
int og_vcycle_precond(int nx, int ny, int nz, double dx, const og_bc* bc, int pin, int num_levels,
                      int pre, int post, int coarse_iters, const double* K, const double* r,
                      double* z) {
    og_hier H;
    og_hier_build(&H, nx, ny, nz, dx, num_levels);
    og_hier_set_K(&H, K);
    og_mgcfg c = {pre, post, coarse_iters};
    og_mg_apply(&H, &c, bc, pin, r, z);
    const int nl = H.nl;
    og_hier_free(&H);
    return nl;
}

/* ------------------------------------------------------------------------ */
/* BLAS-1 (src/numerics/blas) and PCG (src/numerics/solvers/pcg.cuh:95-185)   */
/* ------------------------------------------------------------------------ */
static double og_dot(size_t n, const double* a, const double* b) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

static double og_nrm2(size_t n, const double* a) { return sqrt(og_dot(n, a, a)); }

typedef struct {
    int iterations;
    double initial_residual;
    double final_residual;
    int converged;
    int num_levels;
} og_result;

/* solve_head with solver PCG_MG: src/physics/flow/solve_head.cu:75-234 and pcg.cuh:95-185.
 * If use_guess is 0, h is initialised by init_head_guess; else h holds the initial guess. */
int og_solve_head_pcg(int nx, int ny, int nz, double dx, const og_bc* bc, int pin_mode,
                      int mg_levels, int pre, int post, int coarse_iters, int max_iter,
                      int check_every, double rtol, const double* K, int use_guess, double* h,
                      og_result* res) {
    const size_t n = (size_t)nx * ny * nz;
    int has_dir = 0;
    for (int f = 0; f < 6; ++f) has_dir |= (bc->type[f] == OG_DIRICHLET);
    const int pin = pin_mode == 1 ? 1 : (pin_mode == 2 ? 0 : !has_dir); /* 0 auto, 1 on, 2 off */

    og_hier H;
    og_hier_build(&H, nx, ny, nz, dx, mg_levels);
    og_hier_set_K(&H, K);
    og_mgcfg c = {pre, post, coarse_iters};

    double* b = (double*)malloc(n * sizeof(double));
    double* r = (double*)malloc(n * sizeof(double));
    double* z = (double*)malloc(n * sizeof(double));
    double* p = (double*)malloc(n * sizeof(double));
    double* Ap = (double*)malloc(n * sizeof(double));
    og_build_rhs(nx, ny, nz, dx, bc, K, b);
    if (!use_guess) og_init_guess(nx, ny, nz, bc, h);

    memset(res, 0, sizeof(*res));
    res->num_levels = H.nl;
    og_apply_A(nx, ny, nz, dx, bc, pin, K, h, Ap);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) r[i] = b[i] + (-1.0) * Ap[i];
    res->initial_residual = og_nrm2(n, r);
    if (res->initial_residual < 1e-15) {
        res->converged = 1;
        res->final_residual = res->initial_residual;
        goto done;
    }
    og_mg_apply(&H, &c, bc, pin, r, z);
    memcpy(p, z, n * sizeof(double));
    double rz_old = og_dot(n, r, z);
    for (int it = 0; it < max_iter; ++it) {
        res->iterations = it + 1;
        og_apply_A(nx, ny, nz, dx, bc, pin, K, p, Ap);
        const double pAp = og_dot(n, p, Ap);
        const double alpha = rz_old / pAp;
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < n; ++i) {
            h[i] = h[i] + alpha * p[i];
            r[i] = r[i] + (-alpha) * Ap[i];
        }
        if ((it + 1) % check_every == 0 || it == max_iter - 1) {
            res->final_residual = og_nrm2(n, r);
            if (res->final_residual / res->initial_residual < rtol) {
                res->converged = 1;
                goto done;
            }
        }
        og_mg_apply(&H, &c, bc, pin, r, z);
        const double rz_new = og_dot(n, r, z);
        const double beta = rz_new / rz_old;
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < n; ++i) p[i] = 1.0 * z[i] + beta * p[i];
        rz_old = rz_new;
    }
    res->final_residual = og_nrm2(n, r);
done:
    free(b); free(r); free(z); free(p); free(Ap);
    og_hier_free(&H);
    return 0;
}

/* Standalone MG: solve_head with solver MG, src/multigrid/cycle/v_cycle.cu:76-116
 * (h initialised by init_head_guess, copied into level 0; stop on ||r||/||r0|| < rtol). */
int og_solve_head_mg(int nx, int ny, int nz, double dx, const og_bc* bc, int pin_mode,
                     int mg_levels, int pre, int post, int coarse_iters, int max_cycles,
                     double rtol, const double* K, double* h, og_result* res) {
    const size_t n = (size_t)nx * ny * nz;
    int has_dir = 0;
    for (int f = 0; f < 6; ++f) has_dir |= (bc->type[f] == OG_DIRICHLET);
    const int pin = pin_mode == 1 ? 1 : (pin_mode == 2 ? 0 : !has_dir);
    og_hier H;
    og_hier_build(&H, nx, ny, nz, dx, mg_levels);
    og_hier_set_K(&H, K);
    og_mgcfg c = {pre, post, coarse_iters};
    memset(res, 0, sizeof(*res));
    res->num_levels = H.nl;
    og_build_rhs(nx, ny, nz, dx, bc, K, H.b[0]);
    og_init_guess(nx, ny, nz, bc, h);
    memcpy(H.x[0], h, n * sizeof(double));
    og_residual(nx, ny, nz, dx, bc, pin, H.K[0], H.x[0], H.b[0], H.r[0]);
    res->initial_residual = og_nrm2(n, H.r[0]);
    for (int cyc = 0; cyc < max_cycles; ++cyc) {
        res->iterations = cyc + 1;
        og_vcycle_rec(&H, 0, &c, bc, pin);
        og_residual(nx, ny, nz, dx, bc, pin, H.K[0], H.x[0], H.b[0], H.r[0]);
        res->final_residual = og_nrm2(n, H.r[0]);
        if (res->final_residual / res->initial_residual < rtol) {
            res->converged = 1;
            break;
        }
    }
    memcpy(h, H.x[0], n * sizeof(double));
    og_hier_free(&H);
    return 0;
}

/* Plain CG: solve_head with solver CG, src/physics/flow/solve_head.cu:135-180 and
 * src/numerics/solvers/cg.cuh:14-171: CG on the negated (SPD) operator with rhs -b, x from
 * init_head_guess; stop when ||r|| <= rtol ||r0|| at every check_every-th iteration.  The
 * iterates equal those of CG on A with b (r and p flip sign, alpha is unchanged). */
int og_solve_head_cg(int nx, int ny, int nz, double dx, const og_bc* bc, int pin_mode, int max_iter,
                     int check_every, double rtol, const double* K, double* h, og_result* res) {
    const size_t n = (size_t)nx * ny * nz;
    int has_dir = 0;
    for (int f = 0; f < 6; ++f) has_dir |= (bc->type[f] == OG_DIRICHLET);
    const int pin = pin_mode == 1 ? 1 : (pin_mode == 2 ? 0 : !has_dir);
    double* b = (double*)malloc(n * sizeof(double));
    double* r = (double*)malloc(n * sizeof(double));
    double* p = (double*)malloc(n * sizeof(double));
    double* Ap = (double*)malloc(n * sizeof(double));
    og_build_rhs(nx, ny, nz, dx, bc, K, b);
    og_init_guess(nx, ny, nz, bc, h);
    memset(res, 0, sizeof(*res));
    /* r = (-b) - (-A) x  ==  -(b - A x) */
    og_apply_A(nx, ny, nz, dx, bc, pin, K, h, Ap);
    for (size_t i = 0; i < n; ++i) r[i] = -b[i] + Ap[i];
    memcpy(p, r, n * sizeof(double));
    double rr = og_dot(n, r, r);
    const double r0 = sqrt(rr), tol = r0 * rtol;
    res->initial_residual = r0;
    if (r0 <= tol) {
        res->converged = 1;
        res->final_residual = r0;
        goto done;
    }
    for (int it = 0; it < max_iter; ++it) {
        og_apply_A(nx, ny, nz, dx, bc, pin, K, p, Ap);
        for (size_t i = 0; i < n; ++i) Ap[i] = -Ap[i];
        const double pAp = og_dot(n, p, Ap);
        if ((it + 1) % check_every == 0 && (!(fabs(pAp) >= 1e-30) || !isfinite(pAp))) {
            res->iterations = it + 1;
            res->final_residual = -1.0;
            goto done;
        }
        const double alpha = rr / pAp;
        for (size_t i = 0; i < n; ++i) {
            h[i] += alpha * p[i];
            r[i] -= alpha * Ap[i];
        }
        const double rr_new = og_dot(n, r, r);
        if ((it + 1) % check_every == 0 && sqrt(rr_new) <= tol) {
            res->converged = 1;
            res->iterations = it + 1;
            res->final_residual = sqrt(rr_new);
            goto done;
        }
        const double beta = rr_new / rr;
        for (size_t i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
        rr = rr_new;
    }
    res->iterations = max_iter;
    res->final_residual = sqrt(rr);
done:
    free(b); free(r); free(p); free(Ap);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Face velocity.  src/physics/flow/velocity_from_head.cu:102-551             */
/* layout 0: compact MAC (U (nx+1)*ny*nz, V nx*(ny+1)*nz, W nx*ny*(nz+1));     */
/* layout 1: padded (nx+1)(ny+1)(nz+1) per component, padded_layout.cuh:30.   */
/* Padded entries that are not faces are left untouched.                      */
/* ------------------------------------------------------------------------ */
static inline double og_hm2(double a, double b) { return 2.0 * a * b / (a + b); }

void og_velocity(int nx, int ny, int nz, double dx, const og_bc* bc, const double* H,
                 const double* K, int layout, double* U, double* V, double* W) {
    const double dy = dx, dz = dx;
#define UI(i, j, k) (layout ? ((size_t)(k) * (ny + 1) * (nx + 1) + (size_t)(j) * (nx + 1) + (i)) \
                            : ((size_t)(i) + (size_t)(j) * (nx + 1) + (size_t)(k) * (nx + 1) * ny))
#define VI(i, j, k) (layout ? ((size_t)(k) * (ny + 1) * (nx + 1) + (size_t)(j) * (nx + 1) + (i)) \
                            : ((size_t)(i) + (size_t)(j) * nx + (size_t)(k) * nx * (ny + 1)))
#define WI(i, j, k) (layout ? ((size_t)(k) * (ny + 1) * (nx + 1) + (size_t)(j) * (nx + 1) + (i)) \
                            : ((size_t)(i) + (size_t)(j) * nx + (size_t)(k) * nx * ny))
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) {
            for (int fi = 1; fi <= nx - 1; ++fi) {
                const size_t L = IX(fi - 1, j, k), R = IX(fi, j, k);
                U[UI(fi, j, k)] = -og_hm2(K[L], K[R]) * (H[R] - H[L]) / dx;
            }
            { /* west */
                const size_t c = IX(0, j, k);
                double u = 0.0;
                if (bc->type[0] == OG_DIRICHLET) u = -K[c] * (H[c] - bc->value[0]) / (dx * 0.5);
                else if (bc->type[0] == OG_PERIODIC) {
                    const size_t w = IX(nx - 1, j, k);
                    u = -og_hm2(K[w], K[c]) * (H[c] - H[w]) / dx;
                }
                U[UI(0, j, k)] = u;
            }
            { /* east */
                const size_t c = IX(nx - 1, j, k);
                double u = 0.0;
                if (bc->type[1] == OG_DIRICHLET) u = -K[c] * (bc->value[1] - H[c]) / (dx * 0.5);
                else if (bc->type[1] == OG_PERIODIC) {
                    const size_t w = IX(0, j, k);
                    u = -og_hm2(K[c], K[w]) * (H[w] - H[c]) / dx;
                }
                U[UI(nx, j, k)] = u;
            }
        }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int i = 0; i < nx; ++i) {
            for (int fj = 1; fj <= ny - 1; ++fj) {
                const size_t S = IX(i, fj - 1, k), N = IX(i, fj, k);
                V[VI(i, fj, k)] = -og_hm2(K[S], K[N]) * (H[N] - H[S]) / dy;
            }
            {
                const size_t c = IX(i, 0, k);
                double v = 0.0;
                if (bc->type[2] == OG_DIRICHLET) v = -K[c] * (H[c] - bc->value[2]) / (dy * 0.5);
                else if (bc->type[2] == OG_PERIODIC) {
                    const size_t w = IX(i, ny - 1, k);
                    v = -og_hm2(K[w], K[c]) * (H[c] - H[w]) / dy;
                }
                V[VI(i, 0, k)] = v;
            }
            {
                const size_t c = IX(i, ny - 1, k);
                double v = 0.0;
                if (bc->type[3] == OG_DIRICHLET) v = -K[c] * (bc->value[3] - H[c]) / (dy * 0.5);
                else if (bc->type[3] == OG_PERIODIC) {
                    const size_t w = IX(i, 0, k);
                    v = -og_hm2(K[c], K[w]) * (H[w] - H[c]) / dy;
                }
                V[VI(i, ny, k)] = v;
            }
        }
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            for (int fk = 1; fk <= nz - 1; ++fk) {
                const size_t Bo = IX(i, j, fk - 1), T = IX(i, j, fk);
                W[WI(i, j, fk)] = -og_hm2(K[Bo], K[T]) * (H[T] - H[Bo]) / dz;
            }
            {
                const size_t c = IX(i, j, 0);
                double w = 0.0;
                if (bc->type[4] == OG_DIRICHLET) w = -K[c] * (H[c] - bc->value[4]) / (dz * 0.5);
                else if (bc->type[4] == OG_PERIODIC) {
                    const size_t q = IX(i, j, nz - 1);
                    w = -og_hm2(K[q], K[c]) * (H[c] - H[q]) / dz;
                }
                W[WI(i, j, 0)] = w;
            }
            {
                const size_t c = IX(i, j, nz - 1);
                double w = 0.0;
                if (bc->type[5] == OG_DIRICHLET) w = -K[c] * (bc->value[5] - H[c]) / (dz * 0.5);
                else if (bc->type[5] == OG_PERIODIC) {
                    const size_t q = IX(i, j, 0);
                    w = -og_hm2(K[c], K[q]) * (H[q] - H[c]) / dz;
                }
                W[WI(i, j, nz)] = w;
            }
        }
#undef UI
#undef VI
#undef WI
}

/* Per-cell divergence (compact MAC layout) and the x-face fluxes, for the mass
 * balance check: div_c = sum_f (q_out - q_in) * A_f with A_f = dx^2.
 * Returns max |div_c| in out[0], Q_in (x=0 face) in out[1], Q_out (x=L) in out[2]. */
void og_mass_balance(int nx, int ny, int nz, double dx, const double* U, const double* V,
                     const double* W, double* div, double* out) {
    const double A = dx * dx;
    double mx = 0.0, qin = 0.0, qout = 0.0;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) {
            qin += U[(size_t)0 + (size_t)j * (nx + 1) + (size_t)k * (nx + 1) * ny] * A;
            qout += U[(size_t)nx + (size_t)j * (nx + 1) + (size_t)k * (nx + 1) * ny] * A;
            for (int i = 0; i < nx; ++i) {
                const double du = U[(size_t)(i + 1) + (size_t)j * (nx + 1) + (size_t)k * (nx + 1) * ny] -
                                  U[(size_t)i + (size_t)j * (nx + 1) + (size_t)k * (nx + 1) * ny];
                const double dv = V[(size_t)i + (size_t)(j + 1) * nx + (size_t)k * nx * (ny + 1)] -
                                  V[(size_t)i + (size_t)j * nx + (size_t)k * nx * (ny + 1)];
                const double dw = W[(size_t)i + (size_t)j * nx + (size_t)(k + 1) * nx * ny] -
                                  W[(size_t)i + (size_t)j * nx + (size_t)k * nx * ny];
                const double d = (du + dv + dw) * A;
                if (div) div[IX(i, j, k)] = d;
                if (fabs(d) > mx) mx = fabs(d);
            }
        }
    out[0] = mx;
    out[1] = qin;
    out[2] = qout;
}

/* ------------------------------------------------------------------------ */
/* lnK by the randomization method, given the modes                           */
/* src/physics/stochastic/stochastic.cu:180-205: at cell centres              */
/* lnK = sigma/sqrt(N) * sum_m (a_m sin(k_m.x) + b_m cos(k_m.x)).             */
/* ------------------------------------------------------------------------ */
void og_lnk_eval(int nx, int ny, int nz, double dx, int n_modes, const double* k1,
                 const double* k2, const double* k3, const double* a, const double* b,
                 double sigma, double* lnk) {
    const double scale = sigma / sqrt((double)n_modes);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double x = dx * (i + 0.5), y = dx * (j + 0.5), z = dx * (k + 0.5);
                double s = 0.0;
                for (int m = 0; m < n_modes; ++m) {
                    const double ph = k1[m] * x + k2[m] * y + k3[m] * z;
                    s += a[m] * sin(ph) + b[m] * cos(ph);
                }
                lnk[IX(i, j, k)] = scale * s;
            }
}

/* ------------------------------------------------------------------------ */
/* Randomization-method modes on the host, and lnK evaluated in x-runs.       */
/*                                                                            */
/* The reference draws its modes with cuRAND XORWOW (stochastic.cu:43-91) and */
/* is isotropic; the product draws them with Philox4x32-10 (Salmon, Moraes,   */
/* Dror, Shaw, SC'11), counter (mode, draw, 0, 0), key = seed, and divides    */
/* each wavenumber component by its own correlation length.  This is a        */
/* restatement of that published sampler so that a process that must not load */
/* the product (the reference arm of the bench) can build the same K field.   */
/* The wavenumber magnitude follows stochastic.cu:70-83 (exponential:         */
/* half-Cauchy proposal accepted with k^2/(1+k^2)) and :118-160 (Gaussian).   */
/* ------------------------------------------------------------------------ */
static void og_philox(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t out[4]) {
    uint32_t c[4] = {c0, c1, 0u, 0u};
    uint32_t k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k[0];
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k[1];
        c[1] = (uint32_t)p1;
        c[3] = (uint32_t)p0;
        c[0] = n0;
        c[2] = n2;
        k[0] += 0x9E3779B9u;
        k[1] += 0xBB67AE85u;
    }
    memcpy(out, c, sizeof c);
}

typedef struct {
    uint64_t seed;
    uint32_t mode, draw;
    uint32_t buf[4];
    int have;
} og_mode_rng;

/* 53 random bits from two words, as a double strictly inside (0, 1) */
static double og_u01(og_mode_rng* g) {
    if (g->have == 0) {
        og_philox(g->seed, g->mode, g->draw++, g->buf);
        g->have = 2;
    }
    const uint32_t a = g->have == 2 ? g->buf[0] : g->buf[2];
    const uint32_t b = g->have == 2 ? g->buf[1] : g->buf[3];
    --g->have;
    const uint64_t v = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
    return ((double)v + 0.5) / 9007199254740992.0;
}

/* cov: 0 exponential, 1 Gaussian.  modes: k1, k2, k3, a, b as 5 arrays of n_modes. */
int og_kfield_modes(uint64_t seed, int n_modes, int cov, double lx, double ly, double lz,
                    double* modes) {
    if (n_modes <= 0 || !(lx > 0 && ly > 0 && lz > 0) || (cov != 0 && cov != 1)) return -1;
    const double PI = 3.14159265358979323846;
    double* k1 = modes;
    double* k2 = modes + n_modes;
    double* k3 = modes + 2 * (size_t)n_modes;
    double* am = modes + 3 * (size_t)n_modes;
    double* bm = modes + 4 * (size_t)n_modes;
    for (int m = 0; m < n_modes; ++m) {
        og_mode_rng g = {seed, (uint32_t)m, 0u, {0u, 0u, 0u, 0u}, 0};
        const double fi = 2.0 * PI * og_u01(&g);
        const double theta = acos(1.0 - 2.0 * og_u01(&g));
        double kk = 0.0;
        if (cov == 0) {
            for (int tries = 0; tries < 100000; ++tries) {
                kk = tan(PI * 0.5 * og_u01(&g));
                if (og_u01(&g) < kk * kk / (1.0 + kk * kk)) break;
            }
        } else {
            for (int tries = 0; tries < 100000; ++tries) {
                kk = 10.0 * og_u01(&g);
                if (og_u01(&g) * 2.0 * exp(-1.0) < kk * kk * exp(-0.5 * kk * kk)) break;
            }
            kk *= sqrt(2.0);
        }
        k1[m] = kk * sin(fi) * sin(theta) / lx;
        k2[m] = kk * cos(fi) * sin(theta) / ly;
        k3[m] = kk * cos(theta) / lz;
        double u1 = og_u01(&g), u2 = og_u01(&g);
        am[m] = sqrt(-2.0 * log(u1)) * cos(2.0 * PI * u2);
        u1 = og_u01(&g);
        u2 = og_u01(&g);
        bm[m] = sqrt(-2.0 * log(u1)) * cos(2.0 * PI * u2);
    }
    return 0;
}

/* lnK (want_exp = 0) or K = exp(lnK + log_kg) (want_exp = 1) at cell centres, evaluated as   */
/* the product does: per run of SEG cells along x, sin/cos of the run's first phase, then   */
/* the phase advanced by a rotation through k_x*dx per cell.  Fast enough for 256^3 fields   */
/* on the host; og_lnk_eval above is the direct per-cell form.                              */
void og_kfield_eval_runs(int nx, int ny, int nz, double dx, int n_modes, const double* modes,
                         double sigma, double log_kg, int want_exp, double* out) {
    enum { SEG = 16 };
    const double* k1 = modes;
    const double* k2 = modes + n_modes;
    const double* k3 = modes + 2 * (size_t)n_modes;
    const double* am = modes + 3 * (size_t)n_modes;
    const double* bm = modes + 4 * (size_t)n_modes;
    const double scale = sigma / sqrt((double)n_modes);
    double* sd = (double*)malloc(2 * sizeof(double) * (size_t)n_modes);
    double* cd = sd + n_modes;
    for (int m = 0; m < n_modes; ++m) {
        sd[m] = sin(k1[m] * dx);
        cd[m] = cos(k1[m] * dx);
    }
    const int nseg = (nx + SEG - 1) / SEG;
#pragma omp parallel for schedule(static)
    for (long long task = 0; task < (long long)ny * nz * nseg; ++task) {
        const int seg = (int)(task % nseg);
        const long long row = task / nseg;
        const int j = (int)(row % ny), k = (int)(row / ny);
        const int i0 = seg * SEG;
        const double x0 = dx * (i0 + 0.5), y = dx * (j + 0.5), z = dx * (k + 0.5);
        double acc[SEG];
        for (int t = 0; t < SEG; ++t) acc[t] = 0.0;
        for (int m = 0; m < n_modes; ++m) {
            const double ph = k1[m] * x0 + k2[m] * y + k3[m] * z;
            double s = sin(ph), c = cos(ph);
            const double a = am[m], b = bm[m];
            for (int t = 0; t < SEG; ++t) {
                acc[t] += a * s + b * c;
                const double s2 = s * cd[m] + c * sd[m];
                c = c * cd[m] - s * sd[m];
                s = s2;
            }
        }
        for (int t = 0; t < SEG && i0 + t < nx; ++t) {
            const double v = scale * acc[t];
            out[IX(i0 + t, j, k)] = want_exp ? exp(v + log_kg) : v;
        }
    }
    free(sd);
}

/* ------------------------------------------------------------------------ */
/* Velocity diagnostics at cell centres                                      */
/* src/physics/flow/velocity_diagnostics.cu:48-141 (kernel) and :147-179      */
/* (host): divergence at every cell; |curl u| and helicity u.curl u from      */
/* centred differences of face-averaged cell velocities at interior cells     */
/* (1 <= i <= nx-2, ...), zero elsewhere and everywhere when a dimension is   */
/* below 3.  layout 1 is the reference's padded layout (padded_layout.cuh:30),*/
/* layout 0 the compact MAC arrays.  stats (9 doubles, may be NULL): min, max,*/
/* mean of div, |omega|, helicity over all cells (the mean as the reference's */
/* compute_field_stats gives it, stochastic.cu:369-415: sum / n).             */
/* ------------------------------------------------------------------------ */
static inline size_t og_ui(int lay, int i, int j, int k, int nx, int ny) {
    return lay ? (size_t)k * (ny + 1) * (nx + 1) + (size_t)j * (nx + 1) + (size_t)i
               : (size_t)i + (size_t)j * (nx + 1) + (size_t)k * (nx + 1) * ny;
}
static inline size_t og_vi(int lay, int i, int j, int k, int nx, int ny) {
    return lay ? (size_t)k * (ny + 1) * (nx + 1) + (size_t)j * (nx + 1) + (size_t)i
               : (size_t)i + (size_t)j * nx + (size_t)k * nx * (ny + 1);
}
static inline size_t og_wi(int lay, int i, int j, int k, int nx, int ny) {
    return lay ? (size_t)k * (ny + 1) * (nx + 1) + (size_t)j * (nx + 1) + (size_t)i
               : (size_t)i + (size_t)j * nx + (size_t)k * nx * ny;
}

void og_velocity_diagnostics(int nx, int ny, int nz, double dx, int lay, const double* U,
                             const double* V, const double* W, double* div, double* omag,
                             double* hel, double* stats) {
    const double inv = 1.0 / dx, inv2 = 0.5 * inv;
    const int curl = nx >= 3 && ny >= 3 && nz >= 3;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t c = IX(i, j, k);
                const double Ui = U[og_ui(lay, i, j, k, nx, ny)], Uip = U[og_ui(lay, i + 1, j, k, nx, ny)];
                const double Vj = V[og_vi(lay, i, j, k, nx, ny)], Vjp = V[og_vi(lay, i, j + 1, k, nx, ny)];
                const double Wk = W[og_wi(lay, i, j, k, nx, ny)], Wkp = W[og_wi(lay, i, j, k + 1, nx, ny)];
                div[c] = (Uip - Ui) * inv + (Vjp - Vj) * inv + (Wkp - Wk) * inv;
                if (!curl || i < 1 || i > nx - 2 || j < 1 || j > ny - 2 || k < 1 || k > nz - 2) {
                    omag[c] = 0.0;
                    hel[c] = 0.0;
                    continue;
                }
#define UC(a, b, d) (0.5 * (U[og_ui(lay, a, b, d, nx, ny)] + U[og_ui(lay, (a) + 1, b, d, nx, ny)]))
#define VC(a, b, d) (0.5 * (V[og_vi(lay, a, b, d, nx, ny)] + V[og_vi(lay, a, (b) + 1, d, nx, ny)]))
#define WC(a, b, d) (0.5 * (W[og_wi(lay, a, b, d, nx, ny)] + W[og_wi(lay, a, b, (d) + 1, nx, ny)]))
                const double uc = 0.5 * (Ui + Uip), vc = 0.5 * (Vj + Vjp), wc = 0.5 * (Wk + Wkp);
                const double dwdy = (WC(i, j + 1, k) - WC(i, j - 1, k)) * inv2;
                const double dvdz = (VC(i, j, k + 1) - VC(i, j, k - 1)) * inv2;
                const double dudz = (UC(i, j, k + 1) - UC(i, j, k - 1)) * inv2;
                const double dwdx = (WC(i + 1, j, k) - WC(i - 1, j, k)) * inv2;
                const double dvdx = (VC(i + 1, j, k) - VC(i - 1, j, k)) * inv2;
                const double dudy = (UC(i, j + 1, k) - UC(i, j - 1, k)) * inv2;
#undef UC
#undef VC
#undef WC
                const double ox = dwdy - dvdz, oy = dudz - dwdx, oz = dvdx - dudy;
                omag[c] = sqrt(ox * ox + oy * oy + oz * oz);
                hel[c] = uc * ox + vc * oy + wc * oz;
            }
    if (stats) {
        const double* f[3] = {div, omag, hel};
        const size_t n = (size_t)nx * ny * nz;
        for (int q = 0; q < 3; ++q) {
            double mn = f[q][0], mx = f[q][0], s = 0.0;
            for (size_t c = 0; c < n; ++c) {
                mn = f[q][c] < mn ? f[q][c] : mn;
                mx = f[q][c] > mx ? f[q][c] : mx;
                s += f[q][c];
            }
            stats[3 * q] = mn;
            stats[3 * q + 1] = mx;
            stats[3 * q + 2] = s / (double)n;
        }
    }
}
