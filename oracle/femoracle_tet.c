/*
 * femoracle_tet.c -- CPU oracle for the tetrahedral partial-assembly apply
 * (TEST INFRASTRUCTURE ONLY: the checker of the GPU tet kernels).
 *
 * Restates, per element and per quadrature point, the loops of
 * crates/assembly/src/partial.rs:85-130 (PAMassOperator::apply) and
 * partial.rs:154-208 (PADiffusionOperator::apply) on Tet4 elements:
 *   simplex_jac (partial.rs:290-299): J columns = x_{c+1} - x_0, det J;
 *   J^-T by cofactors, grad_phys = J^-T grad_ref (xform_grads, :301-309);
 *   y_elem[i] += w |det J| kappa (grad u . grad phi_i)  /  w |det J| rho phi_i u;
 *   scatter y[gd[i]] += y_elem[i].
 * Bases: TetP1 / TetP2 / TetP3 (crates/element/src/lagrange/tet.rs:17-236, barycentric
 * formulas); quadrature: tet_rule (crates/element/src/quadrature.rs:259-376),
 * including the Grundmann-Moller construction with per-level weights solved
 * from the x^{2k} moments exactly as that function does.
 * Element DOFs come from the caller ([E][n_ldof], first 4 = the vertex nodes,
 * as DofManager::build_p1 / build_p2_tet number them).
 */
#include "femoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---- tet_rule --------------------------------------------------------- */
/* all non-negative integer n-vectors with sum s, in the recursion order of
 * quadrature.rs:359-372 (first component outermost, ascending) */
static int simplex_points(int s, int n, int (*out)[4], int cap) {
    if (n == 1) {
        if (cap < 1) return 0;
        out[0][0] = s;
        return 1;
    }
    int cnt = 0;
    for (int j0 = 0; j0 <= s; ++j0) {
        int tmp[64][4];
        int m = simplex_points(s - j0, n - 1, tmp, 64);
        for (int k = 0; k < m && cnt < cap; ++k) {
            out[cnt][0] = j0;
            for (int q = 0; q < n - 1; ++q) out[cnt][q + 1] = tmp[k][q];
            ++cnt;
        }
    }
    return cnt;
}

static double fact(int n) {
    double f = 1.0;
    for (int k = 2; k <= n; ++k) f *= k;
    return f;
}

static int grundmann_moller(int s, double *pts, double *w, int cap) {
    const int d = 3, n = s + 1;
    double lv_pts[8][64][3];
    int lv_n[8];
    for (int i = 0; i <= s; ++i) {
        const int si = s - i;
        const double m = 2.0 * si + d + 1;
        int sp[64][4];
        lv_n[i] = simplex_points(si, d + 1, sp, 64);
        for (int k = 0; k < lv_n[i]; ++k)
            for (int c = 0; c < 3; ++c) lv_pts[i][k][c] = (2.0 * sp[k][c + 1] + 1.0) / m;
    }
    /* per-level weights from the x^{2k} moments (Gauss-Jordan with partial pivoting) */
    double mat[8][9];
    for (int k = 0; k < n; ++k) {
        for (int i = 0; i < n; ++i) {
            double sum = 0.0;
            for (int q = 0; q < lv_n[i]; ++q) sum += pow(lv_pts[i][q][0], 2 * k);
            mat[k][i] = sum;
        }
        mat[k][n] = fact(2 * k) / fact(2 * k + 3);
    }
    for (int col = 0; col < n; ++col) {
        int piv = col;
        for (int r = col + 1; r < n; ++r)
            if (fabs(mat[r][col]) > fabs(mat[piv][col])) piv = r;
        if (piv != col)
            for (int j = 0; j <= n; ++j) {
                double t = mat[col][j];
                mat[col][j] = mat[piv][j];
                mat[piv][j] = t;
            }
        const double scale = mat[col][col];
        for (int j = col; j <= n; ++j) mat[col][j] /= scale;
        for (int r = 0; r < n; ++r)
            if (r != col) {
                const double f = mat[r][col];
                for (int j = col; j <= n; ++j) mat[r][j] -= f * mat[col][j];
            }
    }
    int cnt = 0;
    for (int i = 0; i <= s; ++i)
        for (int k = 0; k < lv_n[i] && cnt < cap; ++k) {
            for (int c = 0; c < 3; ++c) pts[3 * cnt + c] = lv_pts[i][k][c];
            w[cnt] = mat[i][n];
            ++cnt;
        }
    return cnt;
}

int or_tet_rule(int order, double *pts, double *w, int cap) {
    if (order <= 1) {
        if (cap < 1) return -1;
        pts[0] = pts[1] = pts[2] = 0.25;
        w[0] = 1.0 / 6.0;
        return 1;
    }
    if (order <= 2) {
        if (cap < 4) return -1;
        const double a = 0.1381966011250105, b = 0.5854101966249685;
        const double p[4][3] = {{a, a, a}, {b, a, a}, {a, b, a}, {a, a, b}};
        for (int q = 0; q < 4; ++q) {
            for (int c = 0; c < 3; ++c) pts[3 * q + c] = p[q][c];
            w[q] = 1.0 / 24.0;
        }
        return 4;
    }
    return grundmann_moller(order <= 5 ? 2 : 3, pts, w, cap);
}

/* ---- TetP1 / TetP2 ----------------------------------------------------- */
int or_tet_basis(int p, const double xi[3], double *phi, double *grad) {
    const double x = xi[0], y = xi[1], z = xi[2];
    const double l1 = 1.0 - x - y - z, l2 = x, l3 = y, l4 = z;
    if (p == 1) {
        phi[0] = l1; phi[1] = l2; phi[2] = l3; phi[3] = l4;
        const double g[12] = {-1, -1, -1, 1, 0, 0, 0, 1, 0, 0, 0, 1};
        memcpy(grad, g, sizeof g);
        return 4;
    }
    if (p == 2) {
        phi[0] = l1 * (2 * l1 - 1); phi[1] = l2 * (2 * l2 - 1);
        phi[2] = l3 * (2 * l3 - 1); phi[3] = l4 * (2 * l4 - 1);
        phi[4] = 4 * l1 * l2; phi[5] = 4 * l1 * l3; phi[6] = 4 * l1 * l4;
        phi[7] = 4 * l2 * l3; phi[8] = 4 * l2 * l4; phi[9] = 4 * l3 * l4;
        const double d0 = 4 * l1 - 1, d1 = 4 * l2 - 1, d2 = 4 * l3 - 1, d3 = 4 * l4 - 1;
        const double g[30] = {-d0, -d0, -d0, d1, 0, 0, 0, d2, 0, 0, 0, d3,
                              4 * (l1 - l2), -4 * l2, -4 * l2,
                              -4 * l3, 4 * (l1 - l3), -4 * l3,
                              -4 * l4, -4 * l4, 4 * (l1 - l4),
                              4 * l3, 4 * l2, 0,
                              4 * l4, 0, 4 * l2,
                              0, 4 * l4, 4 * l3};
        memcpy(grad, g, sizeof g);
        return 10;
    }
    if (p == 3) {
        /* TetP3 (tet.rs:172-236): every basis function is c * prod of factors
         * (alpha * lambda_i + beta); vertices 1/2 l(3l-1)(3l-2), edge DOFs near
         * the first / second vertex 9/2 li lj (3li-1) / (3lj-1), faces 27 li lj lk;
         * gradients by the product rule with grad l1 = (-1,-1,-1), l2..l4 = e_x, e_y, e_z */
        const double L[4] = {l1, l2, l3, l4};
        const double dL[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        int fi[20][3];
        double fa[20][3], fb[20][3], cc[20];
        for (int v = 0; v < 4; ++v) {
            cc[v] = 0.5;
            fi[v][0] = fi[v][1] = fi[v][2] = v;
            fa[v][0] = 1; fb[v][0] = 0; fa[v][1] = 3; fb[v][1] = -1; fa[v][2] = 3; fb[v][2] = -2;
        }
        const int ed[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
        for (int k = 0; k < 6; ++k)
            for (int h = 0; h < 2; ++h) {
                const int d = 4 + 2 * k + h, i = ed[k][0], j = ed[k][1];
                cc[d] = 4.5;
                fi[d][0] = i; fa[d][0] = 1; fb[d][0] = 0;
                fi[d][1] = j; fa[d][1] = 1; fb[d][1] = 0;
                fi[d][2] = h ? j : i; fa[d][2] = 3; fb[d][2] = -1;
            }
        const int fc[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
        for (int k = 0; k < 4; ++k) {
            const int d = 16 + k;
            cc[d] = 27.0;
            for (int m = 0; m < 3; ++m) { fi[d][m] = fc[k][m]; fa[d][m] = 1; fb[d][m] = 0; }
        }
        for (int d = 0; d < 20; ++d) {
            double f[3];
            for (int m = 0; m < 3; ++m) f[m] = fa[d][m] * L[fi[d][m]] + fb[d][m];
            phi[d] = cc[d] * f[0] * f[1] * f[2];
            for (int c = 0; c < 3; ++c)
                grad[3 * d + c] = cc[d] * (fa[d][0] * dL[fi[d][0]][c] * f[1] * f[2] +
                                           f[0] * fa[d][1] * dL[fi[d][1]][c] * f[2] +
                                           f[0] * f[1] * fa[d][2] * dL[fi[d][2]][c]);
        }
        return 20;
    }
    return -1;
}

/* ---- element loop ------------------------------------------------------ */
#define TMAXL 20
#define TMAXQ 64

static void tet_jac(const double *coords, const int32_t *nd, double J[3][3], double *det) {
    const double *x0 = coords + 3 * (int64_t)nd[0];
    for (int c = 0; c < 3; ++c) {
        const double *xc = coords + 3 * (int64_t)nd[c + 1];
        for (int r = 0; r < 3; ++r) J[r][c] = xc[r] - x0[r];
    }
    *det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

static void inv_T(double J[3][3], double det, double jit[3][3]) {
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
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) jit[r][c] = inv[c][r];
}

/* y_e = A_e x_e for one element (kind bits: 1 mass, 2 diffusion) */
static int tet_element(int p, int kind, double c_m, double c_k, const double *coords, const int32_t *gd,
                       int64_t e, const double *kappa_q, double kappa_c, const double *rho_q, double rho_c,
                       int nq, const double *qp, const double *qw, const double *xe, double *ye) {
    double J[3][3], det, jit[3][3];
    tet_jac(coords, gd, J, &det);
    if (!(fabs(det) > 0.0)) return -1;
    inv_T(J, det, jit);
    const int n = p == 1 ? 4 : (p == 2 ? 10 : 20);
    for (int i = 0; i < n; ++i) ye[i] = 0.0;
    for (int q = 0; q < nq; ++q) {
        double phi[TMAXL], gr[3 * TMAXL], gp[3 * TMAXL];
        or_tet_basis(p, qp + 3 * q, phi, gr);
        const double w = qw[q] * fabs(det);
        if (kind & 2) {
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < 3; ++j) {
                    double s = 0.0;
                    for (int k = 0; k < 3; ++k) s += jit[j][k] * gr[3 * i + k];
                    gp[3 * i + j] = s;
                }
            const double kap = c_k * (kappa_q ? kappa_q[e * nq + q] : kappa_c);
            double gu[3] = {0, 0, 0};
            for (int d = 0; d < 3; ++d)
                for (int j = 0; j < n; ++j) gu[d] += xe[j] * gp[3 * j + d];
            for (int i = 0; i < n; ++i) {
                const double dot = gu[0] * gp[3 * i] + gu[1] * gp[3 * i + 1] + gu[2] * gp[3 * i + 2];
                ye[i] += w * kap * dot;
            }
        }
        if (kind & 1) {
            const double rho = c_m * (rho_q ? rho_q[e * nq + q] : rho_c);
            double ux = 0.0;
            for (int j = 0; j < n; ++j) ux += phi[j] * xe[j];
            for (int i = 0; i < n; ++i) ye[i] += w * rho * phi[i] * ux;
        }
    }
    return 0;
}

int or_tet_pa_apply(int p, int64_t n_dofs, const double *coords, int64_t n_elem, const int32_t *elem_dofs,
                    int kind, double c_m, double c_k, const double *kappa_q, double kappa_c,
                    const double *rho_q, double rho_c, int quad_order, const uint8_t *ess,
                    const double *x, double *y, int accumulate) {
    if (p < 1 || p > 3) return -1;
    double qp[3 * TMAXQ], qw[TMAXQ];
    const int nq = or_tet_rule(quad_order, qp, qw, TMAXQ);
    if (nq <= 0) return -1;
    const int n = p == 1 ? 4 : (p == 2 ? 10 : 20);
    if (!accumulate) memset(y, 0, sizeof(double) * n_dofs);
    for (int64_t e = 0; e < n_elem; ++e) {
        const int32_t *gd = elem_dofs + e * n;
        double xe[TMAXL], ye[TMAXL];
        for (int i = 0; i < n; ++i) xe[i] = (ess && ess[gd[i]]) ? 0.0 : x[gd[i]];
        if (tet_element(p, kind, c_m, c_k, coords, gd, e, kappa_q, kappa_c, rho_q, rho_c, nq, qp, qw, xe, ye))
            return -2;
        for (int i = 0; i < n; ++i)
            if (!(ess && ess[gd[i]])) y[gd[i]] += ye[i];
    }
    if (ess)
        for (int64_t i = 0; i < n_dofs; ++i)
            if (ess[i]) y[i] += x[i];
    return 0;
}

int or_tet_diagonal(int p, int64_t n_dofs, const double *coords, int64_t n_elem, const int32_t *elem_dofs,
                    int kind, double c_m, double c_k, const double *kappa_q, double kappa_c,
                    const double *rho_q, double rho_c, int quad_order, const uint8_t *ess, double *d) {
    if (p < 1 || p > 3) return -1;
    double qp[3 * TMAXQ], qw[TMAXQ];
    const int nq = or_tet_rule(quad_order, qp, qw, TMAXQ);
    if (nq <= 0) return -1;
    const int n = p == 1 ? 4 : (p == 2 ? 10 : 20);
    memset(d, 0, sizeof(double) * n_dofs);
    for (int64_t e = 0; e < n_elem; ++e) {
        const int32_t *gd = elem_dofs + e * n;
        for (int i = 0; i < n; ++i) {
            double xe[TMAXL] = {0}, ye[TMAXL];
            xe[i] = 1.0;
            if (tet_element(p, kind, c_m, c_k, coords, gd, e, kappa_q, kappa_c, rho_q, rho_c, nq, qp, qw, xe,
                            ye))
                return -2;
            d[gd[i]] += ye[i];
        }
    }
    if (ess)
        for (int64_t i = 0; i < n_dofs; ++i)
            if (ess[i]) d[i] = 1.0;
    return 0;
}

/* ---- linear form and L2 error on tets (crates/assembly/tests/poisson.rs:437-493)
 * f = 3 pi^2 sin(pi x) sin(pi y) sin(pi z); b_i += w |det J| f(x_q) phi_i,
 * x_q = x_0 + J xi; ess rows set to 0. */
static double tet_usin(const double *x) { return sin(M_PI * x[0]) * sin(M_PI * x[1]) * sin(M_PI * x[2]); }

int or_tet_source(int p, int64_t n_dofs, const double *coords, int64_t n_elem, const int32_t *elem_dofs,
                  int quad_order, const uint8_t *ess, double *b) {
    if (p < 1 || p > 3) return -1;
    double qp[3 * TMAXQ], qw[TMAXQ];
    const int nq = or_tet_rule(quad_order, qp, qw, TMAXQ);
    if (nq <= 0) return -1;
    const int n = p == 1 ? 4 : (p == 2 ? 10 : 20);
    memset(b, 0, sizeof(double) * n_dofs);
    for (int64_t e = 0; e < n_elem; ++e) {
        const int32_t *gd = elem_dofs + e * n;
        double J[3][3], det;
        tet_jac(coords, gd, J, &det);
        const double *x0 = coords + 3 * (int64_t)gd[0];
        for (int q = 0; q < nq; ++q) {
            double phi[TMAXL], gr[3 * TMAXL], xp[3];
            or_tet_basis(p, qp + 3 * q, phi, gr);
            for (int r = 0; r < 3; ++r)
                xp[r] = x0[r] + J[r][0] * qp[3 * q] + J[r][1] * qp[3 * q + 1] + J[r][2] * qp[3 * q + 2];
            const double wf = qw[q] * fabs(det) * 3.0 * M_PI * M_PI * tet_usin(xp);
            for (int i = 0; i < n; ++i) b[gd[i]] += wf * phi[i];
        }
    }
    if (ess)
        for (int64_t i = 0; i < n_dofs; ++i)
            if (ess[i]) b[i] = 0.0;
    return 0;
}

double or_tet_l2_error_sin(int p, const double *coords, int64_t n_elem, const int32_t *elem_dofs, int quad_order,
                           const double *u) {
    if (p < 1 || p > 3) return -1.0;
    double qp[3 * TMAXQ], qw[TMAXQ];
    const int nq = or_tet_rule(quad_order, qp, qw, TMAXQ);
    if (nq <= 0) return -1.0;
    const int n = p == 1 ? 4 : (p == 2 ? 10 : 20);
    double err2 = 0.0;
    for (int64_t e = 0; e < n_elem; ++e) {
        const int32_t *gd = elem_dofs + e * n;
        double J[3][3], det;
        tet_jac(coords, gd, J, &det);
        const double *x0 = coords + 3 * (int64_t)gd[0];
        for (int q = 0; q < nq; ++q) {
            double phi[TMAXL], gr[3 * TMAXL], xp[3];
            or_tet_basis(p, qp + 3 * q, phi, gr);
            for (int r = 0; r < 3; ++r)
                xp[r] = x0[r] + J[r][0] * qp[3 * q] + J[r][1] * qp[3 * q + 1] + J[r][2] * qp[3 * q + 2];
            double uh = 0.0;
            for (int i = 0; i < n; ++i) uh += u[gd[i]] * phi[i];
            const double df = uh - tet_usin(xp);
            err2 += qw[q] * fabs(det) * df * df;
        }
    }
    return sqrt(err2);
}
