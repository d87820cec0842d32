/*
 * femoracle.c -- CPU oracle (test infrastructure only; see femoracle.h for the
 * list of reference files each function restates).
 *
 * Parallelism: elements are split into 8 parity colours (ex%2, ey%2, ez%2);
 * elements of one colour share no DOF, so each colour is an OpenMP loop with a
 * plain `y[g] += y_e` scatter.  Colours run in a fixed order, so results do
 * not depend on the thread count.
 */
#include "femoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXD 4
#define MAXL (MAXD * MAXD * MAXD)

/* ---- quadrature.rs:12-32 gauss_legendre_1d ------------------------------ */
void or_gauss_legendre(int n, double *x, double *w) {
    switch (n) {
    case 1: x[0] = 0.0; w[0] = 2.0; break;
    case 2: {
        double a = 1.0 / sqrt(3.0);
        x[0] = -a; x[1] = a; w[0] = 1.0; w[1] = 1.0;
    } break;
    case 3: {
        double a = sqrt(3.0 / 5.0);
        x[0] = -a; x[1] = 0.0; x[2] = a;
        w[0] = 5.0 / 9.0; w[1] = 8.0 / 9.0; w[2] = 5.0 / 9.0;
    } break;
    case 4: {
        double a = sqrt(3.0 / 7.0 - 2.0 / 7.0 * sqrt(6.0 / 5.0));
        double b = sqrt(3.0 / 7.0 + 2.0 / 7.0 * sqrt(6.0 / 5.0));
        double wa = (18.0 + sqrt(30.0)) / 36.0;
        double wb = (18.0 - sqrt(30.0)) / 36.0;
        x[0] = -b; x[1] = -a; x[2] = a; x[3] = b;
        w[0] = wb; w[1] = wa; w[2] = wa; w[3] = wb;
    } break;
    default: x[0] = 0.0; w[0] = 0.0; break;
    }
}

/* ---- quadrature.rs:405-419 hex_rule: n = clamp((order+2)/2, 1, 4) -------- */
int or_hex_rule_points(int order) {
    int n = (order + 2) / 2;
    if (n < 1) n = 1;
    if (n > 4) n = 4;
    return n;
}

/* 1-D Lagrange polynomials through p+1 equispaced nodes on [-1,1]
 * (node k at -1 + 2k/p): quad.rs:92-105 for p = 2 (L0 = x(x-1)/2,
 * L1 = 1-x^2, L2 = x(x+1)/2), hex.rs:27-36 for p = 1 ((1 -+ x)/2). */
void or_lagrange1d(int p, double xi, double *phi, double *dphi) {
    double nodes[MAXD];
    for (int k = 0; k <= p; ++k) nodes[k] = -1.0 + 2.0 * k / p;
    for (int i = 0; i <= p; ++i) {
        double v = 1.0, dv = 0.0;
        for (int j = 0; j <= p; ++j) {
            if (j == i) continue;
            double den = nodes[i] - nodes[j];
            double prod = 1.0 / den;
            for (int m = 0; m <= p; ++m) {
                if (m == i || m == j) continue;
                prod *= (xi - nodes[m]) / (nodes[i] - nodes[m]);
            }
            dv += prod;
            v *= (xi - nodes[j]) / den;
        }
        phi[i] = v;
        dphi[i] = dv;
    }
}

/* ---- hex.rs:27-66 HexQ1 node table and basis ----------------------------- */
static const double Q1N[8][3] = {
    {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
    {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
/* vertex offsets (di,dj,dk) of the HexQ1 nodes in the structured grid */
static const int Q1OFF[8][3] = {
    {0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
    {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

void or_hexq1_basis(const double xi[3], double phi[8], double grad[24]) {
    for (int i = 0; i < 8; ++i) {
        double fx = 1.0 + Q1N[i][0] * xi[0];
        double fy = 1.0 + Q1N[i][1] * xi[1];
        double fz = 1.0 + Q1N[i][2] * xi[2];
        if (phi) phi[i] = 0.125 * fx * fy * fz;
        if (grad) {
            grad[3 * i + 0] = 0.125 * Q1N[i][0] * fy * fz;
            grad[3 * i + 1] = 0.125 * Q1N[i][1] * fx * fz;
            grad[3 * i + 2] = 0.125 * Q1N[i][2] * fx * fy;
        }
    }
}

int64_t or_ndofs(const or_mesh *m) {
    return (int64_t)(m->nx * m->p + 1) * (m->ny * m->p + 1) * (m->nz * m->p + 1);
}

void or_unit_cube_vertices(int nx, int ny, int nz, double *vc) {
    /* simplex.rs:596-604: lexicographic, i fastest, coords i/n */
    int64_t k3 = 0;
    for (int k = 0; k <= nz; ++k)
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i <= nx; ++i) {
                vc[k3++] = (double)i / nx;
                vc[k3++] = (double)j / ny;
                vc[k3++] = (double)k / nz;
            }
}

static void elem_ijk(const or_mesh *m, int64_t e, int *ex, int *ey, int *ez) {
    *ex = (int)(e % m->nx);
    *ey = (int)((e / m->nx) % m->ny);
    *ez = (int)(e / ((int64_t)m->nx * m->ny));
}

/* Local DOF (a,b,c), a fastest -> global lexicographic DOF. */
void or_elem_dofs(const or_mesh *m, int64_t e, int64_t *dofs) {
    int ex, ey, ez, p = m->p, D = p + 1;
    elem_ijk(m, e, &ex, &ey, &ez);
    int64_t NI = (int64_t)m->nx * p + 1, NJ = (int64_t)m->ny * p + 1;
    for (int c = 0; c < D; ++c)
        for (int b = 0; b < D; ++b)
            for (int a = 0; a < D; ++a)
                dofs[(c * D + b) * D + a] =
                    ((int64_t)(ez * p + c) * NJ + (ey * p + b)) * NI + (ex * p + a);
}

static void elem_vertices(const or_mesh *m, int64_t e, double xv[8][3]) {
    int ex, ey, ez;
    elem_ijk(m, e, &ex, &ey, &ez);
    for (int v = 0; v < 8; ++v) {
        int i = ex + Q1OFF[v][0], j = ey + Q1OFF[v][1], k = ez + Q1OFF[v][2];
        if (m->vcoord) {
            int64_t id = ((int64_t)k * (m->ny + 1) + j) * (m->nx + 1) + i;
            xv[v][0] = m->vcoord[3 * id + 0];
            xv[v][1] = m->vcoord[3 * id + 1];
            xv[v][2] = m->vcoord[3 * id + 2];
        } else {
            xv[v][0] = (double)i / m->nx;
            xv[v][1] = (double)j / m->ny;
            xv[v][2] = (double)k / m->nz;
        }
    }
}

/* Tabulated reference element at the quadrature points: the reference
 * re-evaluates the same values per element (partial.rs:182); tabulating once
 * yields identical numbers. */
typedef struct {
    int D, L, nq, Q3;
    double xq[MAXD], wq[MAXD];
    double *phi;   /* [Q3][L] */
    double *gref;  /* [Q3][L][3] */
    double *gq1;   /* [Q3][8][3] Q1 geometry gradients */
    double *pq1;   /* [Q3][8] Q1 geometry values */
    double *w;     /* [Q3] */
} reftab;

static void reftab_init(reftab *t, int p, int nq) {
    t->D = p + 1;
    t->L = t->D * t->D * t->D;
    t->nq = nq;
    t->Q3 = nq * nq * nq;
    or_gauss_legendre(nq, t->xq, t->wq);
    t->phi = (double *)malloc(sizeof(double) * t->Q3 * t->L);
    t->gref = (double *)malloc(sizeof(double) * t->Q3 * t->L * 3);
    t->gq1 = (double *)malloc(sizeof(double) * t->Q3 * 24);
    t->pq1 = (double *)malloc(sizeof(double) * t->Q3 * 8);
    t->w = (double *)malloc(sizeof(double) * t->Q3);
    int D = t->D;
    for (int kz = 0; kz < nq; ++kz)
        for (int ky = 0; ky < nq; ++ky)
            for (int kx = 0; kx < nq; ++kx) {
                int q = (kz * nq + ky) * nq + kx;
                double xi[3] = {t->xq[kx], t->xq[ky], t->xq[kz]};
                double Lx[MAXD], dLx[MAXD], Ly[MAXD], dLy[MAXD], Lz[MAXD], dLz[MAXD];
                or_lagrange1d(p, xi[0], Lx, dLx);
                or_lagrange1d(p, xi[1], Ly, dLy);
                or_lagrange1d(p, xi[2], Lz, dLz);
                for (int c = 0; c < D; ++c)
                    for (int b = 0; b < D; ++b)
                        for (int a = 0; a < D; ++a) {
                            int i = (c * D + b) * D + a;
                            t->phi[q * t->L + i] = Lx[a] * Ly[b] * Lz[c];
                            t->gref[(q * t->L + i) * 3 + 0] = dLx[a] * Ly[b] * Lz[c];
                            t->gref[(q * t->L + i) * 3 + 1] = Lx[a] * dLy[b] * Lz[c];
                            t->gref[(q * t->L + i) * 3 + 2] = Lx[a] * Ly[b] * dLz[c];
                        }
                or_hexq1_basis(xi, t->pq1 + 8 * q, t->gq1 + 24 * q);
                t->w[q] = t->wq[kx] * t->wq[ky] * t->wq[kz];
            }
}

static void reftab_free(reftab *t) {
    free(t->phi); free(t->gref); free(t->gq1); free(t->pq1); free(t->w);
}

/* assembler.rs:96-123 isoparametric_jacobian: J_id = sum_k x_k[i] dphi_k/dxi_d */
static double iso_jacobian(const double xv[8][3], const double *g, const double *pv,
                           double J[3][3], double xp[3]) {
    memset(J, 0, sizeof(double) * 9);
    xp[0] = xp[1] = xp[2] = 0.0;
    for (int k = 0; k < 8; ++k)
        for (int i = 0; i < 3; ++i) {
            xp[i] += pv[k] * xv[k][i];
            for (int d = 0; d < 3; ++d) J[i][d] += xv[k][i] * g[3 * k + d];
        }
    return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
           J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

/* J^{-T} (the `jit` of assembler.rs:224-226) */
static void inv_transpose(double J[3][3], double det, double jit[3][3]) {
    double inv[3][3];
    inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
    inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
    inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
    inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
    inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
    inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
    inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
    inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
    inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) jit[i][j] = inv[j][i];
}

typedef struct {
    int kind;
    double c_m, c_k;
    const double *kappa_q, *rho_q;
    double kappa_c, rho_c;
} coefs;

/* One element of partial.rs:154-208 (diffusion) and :85-130 (mass):
 * per quadrature point transform the reference gradients by J^{-T},
 * grad u = sum_j x_j grad phi_j, y_e[i] += w kappa grad u . grad phi_i. */
static void element_apply(const or_mesh *m, const reftab *t, const coefs *cf, int64_t e,
                          const double *xe, double *ye) {
    double xv[8][3];
    elem_vertices(m, e, xv);
    int L = t->L;
    double gphys[MAXL * 3];
    for (int i = 0; i < L; ++i) ye[i] = 0.0;
    for (int q = 0; q < t->Q3; ++q) {
        double J[3][3], xp[3], jit[3][3];
        double det = iso_jacobian(xv, t->gq1 + 24 * q, t->pq1 + 8 * q, J, xp);
        double w = t->w[q] * fabs(det);
        if (cf->kind & OR_DIFF) {
            inv_transpose(J, det, jit);
            const double *gr = t->gref + (size_t)q * L * 3;
            for (int i = 0; i < L; ++i)
                for (int j = 0; j < 3; ++j) {
                    double s = 0.0;
                    for (int k = 0; k < 3; ++k) s += jit[j][k] * gr[3 * i + k];
                    gphys[3 * i + j] = s;
                }
            double kap = cf->kappa_q ? cf->kappa_q[e * t->Q3 + q] : cf->kappa_c;
            double gu[3] = {0, 0, 0};
            for (int j = 0; j < L; ++j)
                for (int d = 0; d < 3; ++d) gu[d] += xe[j] * gphys[3 * j + d];
            double s = w * kap * cf->c_k;
            for (int i = 0; i < L; ++i) {
                double dot = gu[0] * gphys[3 * i] + gu[1] * gphys[3 * i + 1] + gu[2] * gphys[3 * i + 2];
                ye[i] += s * dot;
            }
        }
        if (cf->kind & OR_MASS) {
            const double *ph = t->phi + (size_t)q * L;
            double rho = cf->rho_q ? cf->rho_q[e * t->Q3 + q] : cf->rho_c;
            double ux = 0.0;
            for (int j = 0; j < L; ++j) ux += ph[j] * xe[j];
            double s = w * rho * cf->c_m * ux;
            for (int i = 0; i < L; ++i) ye[i] += s * ph[i];
        }
    }
}

static void element_diag(const or_mesh *m, const reftab *t, const coefs *cf, int64_t e,
                         double *de) {
    double xv[8][3];
    elem_vertices(m, e, xv);
    int L = t->L;
    for (int i = 0; i < L; ++i) de[i] = 0.0;
    for (int q = 0; q < t->Q3; ++q) {
        double J[3][3], xp[3], jit[3][3];
        double det = iso_jacobian(xv, t->gq1 + 24 * q, t->pq1 + 8 * q, J, xp);
        double w = t->w[q] * fabs(det);
        if (cf->kind & OR_DIFF) {
            inv_transpose(J, det, jit);
            const double *gr = t->gref + (size_t)q * L * 3;
            double kap = cf->kappa_q ? cf->kappa_q[e * t->Q3 + q] : cf->kappa_c;
            for (int i = 0; i < L; ++i) {
                double g2 = 0.0;
                for (int j = 0; j < 3; ++j) {
                    double s = 0.0;
                    for (int k = 0; k < 3; ++k) s += jit[j][k] * gr[3 * i + k];
                    g2 += s * s;
                }
                de[i] += w * kap * cf->c_k * g2;
            }
        }
        if (cf->kind & OR_MASS) {
            const double *ph = t->phi + (size_t)q * L;
            double rho = cf->rho_q ? cf->rho_q[e * t->Q3 + q] : cf->rho_c;
            for (int i = 0; i < L; ++i) de[i] += w * rho * cf->c_m * ph[i] * ph[i];
        }
    }
}

static int set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
    return omp_get_max_threads();
#else
    (void)nthreads;
    return 1;
#endif
}

/* Coloured element loop: colour = (ex&1) | (ey&1)<<1 | (ez&1)<<2. */
#define FOR_COLOURED_ELEMENTS(m, ...)                                              \
    for (int colour = 0; colour < 8; ++colour) {                                    \
        int cx = colour & 1, cy = (colour >> 1) & 1, cz = (colour >> 2) & 1;        \
        int hx = (m->nx - cx + 1) / 2, hy = (m->ny - cy + 1) / 2, hz = (m->nz - cz + 1) / 2; \
        int64_t ncol = (int64_t)hx * hy * hz;                                       \
        _Pragma("omp parallel for schedule(static)")                                \
        for (int64_t ic = 0; ic < ncol; ++ic) {                                     \
            int ix = (int)(ic % hx), iy = (int)((ic / hx) % hy), iz = (int)(ic / ((int64_t)hx * hy)); \
            int64_t e = ((int64_t)(2 * iz + cz) * m->ny + (2 * iy + cy)) * m->nx + (2 * ix + cx); \
            __VA_ARGS__                                                             \
        }                                                                           \
    }

static int apply_impl(const or_mesh *m, const coefs *cf, const uint8_t *ess,
                      const double *x, double *y, int accumulate, int nthreads) {
    if (m->p < 1 || m->p > 3 || m->nq < 1 || m->nq > 4) return 4;
    set_threads(nthreads);
    int64_t N = or_ndofs(m);
    if (!accumulate) memset(y, 0, sizeof(double) * N);
    reftab t;
    reftab_init(&t, m->p, m->nq);
    int L = t.L;
    FOR_COLOURED_ELEMENTS(m, {
        int64_t dofs[MAXL];
        double xe[MAXL], ye[MAXL];
        or_elem_dofs(m, e, dofs);
        for (int i = 0; i < L; ++i) xe[i] = (ess && ess[dofs[i]]) ? 0.0 : x[dofs[i]];
        element_apply(m, &t, cf, e, xe, ye);
        for (int i = 0; i < L; ++i) y[dofs[i]] += ye[i];
    })
    if (ess) {
        for (int64_t i = 0; i < N; ++i)
            if (ess[i]) y[i] = accumulate ? y[i] + x[i] : x[i];
    }
    reftab_free(&t);
    return 0;
}

int or_pa_apply(const or_mesh *m, int kind, double c_m, double c_k,
                const double *kappa_q, double kappa_c, const double *rho_q, double rho_c,
                const double *x, double *y, int accumulate, int nthreads) {
    coefs cf = {kind, c_m, c_k, kappa_q, rho_q, kappa_c, rho_c};
    return apply_impl(m, &cf, NULL, x, y, accumulate, nthreads);
}

int or_apply_constrained(const or_mesh *m, int kind, double c_m, double c_k,
                         const double *kappa_q, double kappa_c, const double *rho_q,
                         double rho_c, const uint8_t *ess, const double *x, double *y,
                         int nthreads) {
    coefs cf = {kind, c_m, c_k, kappa_q, rho_q, kappa_c, rho_c};
    return apply_impl(m, &cf, ess, x, y, 0, nthreads);
}

int or_element_matrix(const or_mesh *m, int64_t e, int kind, double c_m, double c_k,
                      const double *kappa_q, double kappa_c, const double *rho_q,
                      double rho_c, double *Ke) {
    coefs cf = {kind, c_m, c_k, kappa_q, rho_q, kappa_c, rho_c};
    reftab t;
    reftab_init(&t, m->p, m->nq);
    int L = t.L;
    double xe[MAXL], ye[MAXL];
    for (int j = 0; j < L; ++j) {
        for (int i = 0; i < L; ++i) xe[i] = (i == j) ? 1.0 : 0.0;
        element_apply(m, &t, &cf, e, xe, ye);
        for (int i = 0; i < L; ++i) Ke[i * L + j] = ye[i];
    }
    reftab_free(&t);
    return 0;
}

void or_ess_mask(const or_mesh *m, int tag_bits, uint8_t *mask) {
    int p = m->p;
    int64_t NI = (int64_t)m->nx * p + 1, NJ = (int64_t)m->ny * p + 1, NK = (int64_t)m->nz * p + 1;
    for (int64_t K = 0; K < NK; ++K)
        for (int64_t J = 0; J < NJ; ++J)
            for (int64_t I = 0; I < NI; ++I) {
                int on = ((tag_bits & 1) && K == 0) || ((tag_bits & 2) && K == NK - 1) ||
                         ((tag_bits & 4) && J == 0) || ((tag_bits & 8) && J == NJ - 1) ||
                         ((tag_bits & 16) && I == 0) || ((tag_bits & 32) && I == NI - 1);
                mask[(K * NJ + J) * NI + I] = (uint8_t)on;
            }
}

int or_diagonal(const or_mesh *m, int kind, double c_m, double c_k,
                const double *kappa_q, double kappa_c, const double *rho_q, double rho_c,
                const uint8_t *ess, double *d, int nthreads) {
    coefs cf = {kind, c_m, c_k, kappa_q, rho_q, kappa_c, rho_c};
    set_threads(nthreads);
    int64_t N = or_ndofs(m);
    memset(d, 0, sizeof(double) * N);
    reftab t;
    reftab_init(&t, m->p, m->nq);
    int L = t.L;
    FOR_COLOURED_ELEMENTS(m, {
        int64_t dofs[MAXL];
        double de[MAXL];
        or_elem_dofs(m, e, dofs);
        element_diag(m, &t, &cf, e, de);
        for (int i = 0; i < L; ++i) d[dofs[i]] += de[i];
    })
    if (ess)
        for (int64_t i = 0; i < N; ++i)
            if (ess[i]) d[i] = 1.0;
    reftab_free(&t);
    return 0;
}

static double f_sin(const double x[3]) {
    const double pi = 3.14159265358979323846;
    return 3.0 * pi * pi * sin(pi * x[0]) * sin(pi * x[1]) * sin(pi * x[2]);
}
static double u_sin(const double x[3]) {
    const double pi = 3.14159265358979323846;
    return sin(pi * x[0]) * sin(pi * x[1]) * sin(pi * x[2]);
}

/* standard/source.rs:39-50: f_elem[i] += w f(x) phi_i; assembler.rs:434-454 */
int or_source(const or_mesh *m, int f_kind, int nq, const uint8_t *ess, double *b) {
    (void)f_kind;
    if (nq < 1 || nq > MAXD) return -1; /* hex_rule clamps to 4 points (quadrature.rs:405-419) */
    int64_t N = or_ndofs(m);
    memset(b, 0, sizeof(double) * N);
    reftab t;
    reftab_init(&t, m->p, nq);
    int L = t.L;
    FOR_COLOURED_ELEMENTS(m, {
        int64_t dofs[MAXL];
        double xv[8][3], fe[MAXL];
        or_elem_dofs(m, e, dofs);
        elem_vertices(m, e, xv);
        for (int i = 0; i < L; ++i) fe[i] = 0.0;
        for (int q = 0; q < t.Q3; ++q) {
            double J[3][3], xp[3];
            double det = iso_jacobian(xv, t.gq1 + 24 * q, t.pq1 + 8 * q, J, xp);
            double wf = t.w[q] * fabs(det) * f_sin(xp);
            for (int i = 0; i < L; ++i) fe[i] += wf * t.phi[q * L + i];
        }
        for (int i = 0; i < L; ++i) b[dofs[i]] += fe[i];
    })
    if (ess)
        for (int64_t i = 0; i < N; ++i)
            if (ess[i]) b[i] = 0.0;
    reftab_free(&t);
    return 0;
}

/* partial.rs:222-248 (LumpedMassOperator::assemble) on hexahedra: per
 * quadrature point diag_i += w |det J| rho phi_i (sum_j phi_j). */
int or_lumped_mass(const or_mesh *m, const double *rho_q, double rho_c, int nq, double *diag) {
    if (nq < 1 || nq > MAXD) return -1;
    int64_t N = or_ndofs(m);
    memset(diag, 0, sizeof(double) * N);
    reftab t;
    reftab_init(&t, m->p, nq);
    int L = t.L;
    FOR_COLOURED_ELEMENTS(m, {
        int64_t dofs[MAXL];
        double xv[8][3], de[MAXL];
        or_elem_dofs(m, e, dofs);
        elem_vertices(m, e, xv);
        for (int i = 0; i < L; ++i) de[i] = 0.0;
        for (int q = 0; q < t.Q3; ++q) {
            double J[3][3], xp[3];
            double det = iso_jacobian(xv, t.gq1 + 24 * q, t.pq1 + 8 * q, J, xp);
            double rho = rho_q ? rho_q[e * t.Q3 + q] : rho_c;
            double w = t.w[q] * fabs(det);
            double psum = 0.0;
            for (int j = 0; j < L; ++j) psum += t.phi[q * L + j];
            for (int i = 0; i < L; ++i) de[i] += w * rho * t.phi[q * L + i] * psum;
        }
        for (int i = 0; i < L; ++i) diag[dofs[i]] += de[i];
    })
    reftab_free(&t);
    return 0;
}

double or_l2_error_sin(const or_mesh *m, int nq, const double *u) {
    if (nq < 1 || nq > MAXD) return -1.0;
    reftab t;
    reftab_init(&t, m->p, nq);
    int L = t.L;
    int64_t E = (int64_t)m->nx * m->ny * m->nz;
    /* fixed element chunks summed in index order: the same result on any
     * thread count (see dot() below) */
    double part[64];
#pragma omp parallel for schedule(static)
    for (int c = 0; c < 64; ++c) {
        double err2 = 0.0;
        for (int64_t e = E * c / 64; e < E * (c + 1) / 64; ++e) {
            int64_t dofs[MAXL];
            double xv[8][3];
            or_elem_dofs(m, e, dofs);
            elem_vertices(m, e, xv);
            for (int q = 0; q < t.Q3; ++q) {
                double J[3][3], xp[3];
                double det = iso_jacobian(xv, t.gq1 + 24 * q, t.pq1 + 8 * q, J, xp);
                double uh = 0.0;
                for (int i = 0; i < L; ++i) uh += t.phi[q * L + i] * u[dofs[i]];
                double df = uh - u_sin(xp);
                err2 += t.w[q] * fabs(det) * df * df;
            }
        }
        part[c] = err2;
    }
    double err2 = 0.0;
    for (int c = 0; c < 64; ++c) err2 += part[c];
    reftab_free(&t);
    return sqrt(err2);
}

/* ---------------------------------------------------------------------- */
/* Krylov solvers on the constrained operator                             */
/* ---------------------------------------------------------------------- */

/* Dot product with a summation order that does not depend on the thread count
 * or on which thread finishes first (an OpenMP reduction clause combines the
 * per-thread sums in arrival order): fixed chunks, chunk sums added in index
 * order.  The iteration counts of the Krylov solvers below are therefore the
 * same on every host. */
#define OR_DOT_CHUNKS 64
static double dot(int64_t n, const double *a, const double *b) {
    double part[OR_DOT_CHUNKS];
#pragma omp parallel for schedule(static)
    for (int c = 0; c < OR_DOT_CHUNKS; ++c) {
        const int64_t i0 = n * c / OR_DOT_CHUNKS, i1 = n * (c + 1) / OR_DOT_CHUNKS;
        double s = 0.0;
        for (int64_t i = i0; i < i1; ++i) s += a[i] * b[i];
        part[c] = s;
    }
    double s = 0.0;
    for (int c = 0; c < OR_DOT_CHUNKS; ++c) s += part[c];
    return s;
}

typedef struct {
    const or_mesh *m;
    coefs cf;
    const uint8_t *ess;
    int nthreads;
    int64_t applies;
} opctx;

static void op_apply(opctx *o, const double *x, double *y) {
    apply_impl(o->m, &o->cf, o->ess, x, y, 0, o->nthreads);
    o->applies++;
}

/* Deterministic start vector for power iteration: splitmix64 hash of the
 * index mapped to [-1, 1). The CUDA library uses the same sequence. */
static double hash_unit(uint64_t i) {
    uint64_t z = i + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

static double lambda_max_impl(opctx *o, const double *dinv, int64_t N, int iters) {
    double *v = (double *)malloc(sizeof(double) * N);
    double *w = (double *)malloc(sizeof(double) * N);
    for (int64_t i = 0; i < N; ++i) v[i] = hash_unit((uint64_t)i);
    double nv = sqrt(dot(N, v, v));
    for (int64_t i = 0; i < N; ++i) v[i] /= nv;
    double rho = 1.0;
    /* amg/src/lib.rs:108-123: w = A v, rho = ||w||, v = w / rho; here on D^-1 A */
    for (int it = 0; it < iters; ++it) {
        op_apply(o, v, w);
        for (int64_t i = 0; i < N; ++i) w[i] *= dinv[i];
        rho = sqrt(dot(N, w, w));
        if (rho > 1e-14)
            for (int64_t i = 0; i < N; ++i) v[i] = w[i] / rho;
    }
    free(v);
    free(w);
    return rho;
}

/* z = Chebyshev(k)(D^-1 A)^-1-approx applied to r, Saad Alg. 12.1 from z0 = 0 */
static void cheb_apply(opctx *o, const double *dinv, int64_t N, int k, double lmin,
                       double lmax, const double *r, double *z, double *res, double *d,
                       double *tmp) {
    double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
    double sigma = theta / delta, rho = 1.0 / sigma;
    for (int64_t i = 0; i < N; ++i) {
        res[i] = dinv[i] * r[i];
        d[i] = res[i] / theta;
        z[i] = d[i];
    }
    for (int s = 1; s < k; ++s) {
        op_apply(o, d, tmp);
        double rho_new = 1.0 / (2.0 * sigma - rho);
        double c1 = rho_new * rho, c2 = 2.0 * rho_new / delta;
        for (int64_t i = 0; i < N; ++i) {
            res[i] -= dinv[i] * tmp[i];
            d[i] = c1 * d[i] + c2 * res[i];
            z[i] += d[i];
        }
        rho = rho_new;
    }
}

double or_lambda_max(const or_mesh *m, int kind, double c_m, double c_k,
                     const double *kappa_q, double kappa_c, const double *rho_q,
                     double rho_c, const uint8_t *ess, int iters, int nthreads) {
    opctx o = {m, {kind, c_m, c_k, kappa_q, rho_q, kappa_c, rho_c}, ess, nthreads, 0};
    set_threads(nthreads);
    int64_t N = or_ndofs(m);
    double *dg = (double *)malloc(sizeof(double) * N);
    or_diagonal(m, kind, c_m, c_k, kappa_q, kappa_c, rho_q, rho_c, ess, dg, nthreads);
    for (int64_t i = 0; i < N; ++i) dg[i] = fabs(dg[i]) > 1e-30 ? 1.0 / dg[i] : 1.0;
    double l = lambda_max_impl(&o, dg, N, iters);
    free(dg);
    return l;
}

/* par_solver.rs:262-342 (Jacobi) generalised to z = M r; precond 0 is the
 * operator CG of solver/src/lib.rs:198-278 with its own stopping rule
 * (||r|| <= max(atol, rtol*max(||b||, 1e-32)), absolute final residual). */
int or_pcg(const or_mesh *m, int kind, double c_m, double c_k,
           const double *kappa_q, double kappa_c, const double *rho_q, double rho_c,
           const uint8_t *ess, const double *b, double *x, const or_cfg *cfg,
           or_result *res, int nthreads) {
    opctx o = {m, {kind, c_m, c_k, kappa_q, rho_q, kappa_c, rho_c}, ess, nthreads, 0};
    set_threads(nthreads);
    int64_t N = or_ndofs(m);
    double *r = (double *)malloc(sizeof(double) * N);
    double *z = (double *)malloc(sizeof(double) * N);
    double *p = (double *)malloc(sizeof(double) * N);
    double *ap = (double *)malloc(sizeof(double) * N);
    double *dinv = (double *)malloc(sizeof(double) * N);
    double *w1 = NULL, *w2 = NULL, *w3 = NULL;
    memset(res, 0, sizeof(*res));
    or_diagonal(m, kind, c_m, c_k, kappa_q, kappa_c, rho_q, rho_c, ess, dinv, nthreads);
    for (int64_t i = 0; i < N; ++i) dinv[i] = fabs(dinv[i]) > 1e-30 ? 1.0 / dinv[i] : 1.0;
    double lmin = cfg->lmin, lmax = cfg->lmax;
    if (cfg->precond == 2) {
        w1 = (double *)malloc(sizeof(double) * N);
        w2 = (double *)malloc(sizeof(double) * N);
        w3 = (double *)malloc(sizeof(double) * N);
    }
    op_apply(&o, x, ap);
    for (int64_t i = 0; i < N; ++i) r[i] = b[i] - ap[i];
#define PRECOND(src, dst)                                                              \
    do {                                                                               \
        if (cfg->precond == 1)                                                         \
            for (int64_t i_ = 0; i_ < N; ++i_) dst[i_] = dinv[i_] * src[i_];           \
        else if (cfg->precond == 2)                                                    \
            cheb_apply(&o, dinv, N, cfg->cheb_degree, lmin, lmax, src, dst, w1, w2, w3); \
        else                                                                           \
            memcpy(dst, src, sizeof(double) * N);                                      \
    } while (0)
    PRECOND(r, z);
    memcpy(p, z, sizeof(double) * N);
    double rz = dot(N, r, z);
    double bnorm = sqrt(dot(N, b, b));
    int conv = 0, it_done = cfg->max_iter;
    double final_res = 0.0;
    /* precond 0 = solve_cg_operator (lib.rs:229-278): tol = max(atol,
     * rtol*max(||b||, 1e-32)), converged when ||r|| <= tol (checked before the
     * first iteration too), breakdown |pAp| < 1e-32, absolute final residual */
    const int cgop = cfg->precond == 0;
    const double tol_abs = fmax(cfg->atol, cfg->rtol * fmax(bnorm, 1e-32));
    if (cgop) {
        final_res = sqrt(rz);
        if (final_res <= tol_abs) {
            conv = 1; it_done = 0;
            goto done;
        }
    } else if (bnorm < 1e-30) {
        conv = 1; it_done = 0; final_res = 0.0;
        goto done;
    }
    for (int iter = 0; iter < cfg->max_iter; ++iter) {
        op_apply(&o, p, ap);
        double pap = dot(N, p, ap);
        if (fabs(pap) < (cgop ? 1e-32 : 1e-30)) break;
        double alpha = rz / pap;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * ap[i];
        }
        double rr = dot(N, r, r);
        double rn = sqrt(rr) / bnorm;
        final_res = cgop ? sqrt(rr) : rn;
        if (cgop ? sqrt(rr) <= tol_abs : (rn < cfg->rtol || sqrt(rr) < cfg->atol)) {
            conv = 1; it_done = iter + 1;
            goto done;
        }
        PRECOND(r, z);
        double rz_new = dot(N, r, z);
        double beta = rz_new / rz;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) p[i] = z[i] + beta * p[i];
        rz = rz_new;
    }
    final_res = cgop ? sqrt(dot(N, r, r)) : sqrt(dot(N, r, r)) / bnorm;
done:
    res->converged = conv;
    res->iterations = it_done;
    res->final_residual = final_res;
    op_apply(&o, x, ap);
    for (int64_t i = 0; i < N; ++i) ap[i] = b[i] - ap[i];
    res->true_residual = bnorm > 0 ? sqrt(dot(N, ap, ap)) / bnorm : 0.0;
    res->applies = o.applies;
    free(r); free(z); free(p); free(ap); free(dinv);
    free(w1); free(w2); free(w3);
#undef PRECOND
    return conv ? 0 : 1;
}

/* ---- amg/src/lib.rs:53-103, restated verbatim in structure (compat only) -- */
static void csr_spmv(int64_t n, const int64_t *rp, const int64_t *ci, const double *v,
                     const double *x, double *y) {
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
        y[i] = s;
    }
}

void or_ref_chebyshev_smooth_csr(int64_t n, const int64_t *rp, const int64_t *ci,
                                 const double *v, double *x, const double *b,
                                 double lmin, double lmax, int n_iter) {
    double alpha = (lmax + lmin) / 2.0, delta = (lmax - lmin) / 2.0;
    double *dinv = (double *)malloc(sizeof(double) * n);
    double *r = (double *)calloc((size_t)n, sizeof(double));
    double *d = (double *)calloc((size_t)n, sizeof(double));
    for (int64_t i = 0; i < n; ++i) {
        double di = 0.0;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) di = v[k];
        dinv[i] = fabs(di) > 1e-14 ? 1.0 / di : 1.0;
    }
    double two_over_alpha = 2.0 / alpha;
    double q = (delta / (2.0 * alpha)) * (delta / (2.0 * alpha));
    double rho_prev = 0.0;
    for (int k = 0; k < n_iter; ++k) {
        csr_spmv(n, rp, ci, v, x, r);
        for (int64_t i = 0; i < n; ++i) r[i] = b[i] - r[i];
        if (k == 0) {
            for (int64_t i = 0; i < n; ++i) d[i] = two_over_alpha * dinv[i] * r[i];
            rho_prev = 1.0;
        } else {
            double rho = 1.0 / (1.0 - q * rho_prev);
            for (int64_t i = 0; i < n; ++i)
                d[i] = rho * (two_over_alpha * dinv[i] * r[i] + (rho - 1.0) * d[i]);
            rho_prev = rho;
        }
        for (int64_t i = 0; i < n; ++i) x[i] += d[i];
    }
    free(dinv); free(r); free(d);
}

double or_ref_spectral_radius_csr(int64_t n, const int64_t *rp, const int64_t *ci,
                                  const double *v, int n_iter) {
    double *x = (double *)malloc(sizeof(double) * n);
    double *w = (double *)malloc(sizeof(double) * n);
    for (int64_t i = 0; i < n; ++i) x[i] = 1.0 / sqrt((double)n);
    double rho = 1.0;
    for (int it = 0; it < n_iter; ++it) {
        csr_spmv(n, rp, ci, v, x, w);
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) s += w[i] * w[i];
        rho = sqrt(s);
        if (rho > 1e-14)
            for (int64_t i = 0; i < n; ++i) x[i] = w[i] / rho;
    }
    free(x); free(w);
    return rho;
}
