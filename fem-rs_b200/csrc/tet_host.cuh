// tet_host.cuh -- host side of the tetrahedral PA operator (included by
// femgpu.cu, single translation unit).
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <mutex>
#include <vector>

#include "tet_kernels.cuh"

struct fg_tet {
    int device = 0;
    int p = 1, nl = 4, kind = 2;
    int64_t E = 0, N = 0, n_nodes = 0;
    int32_t *dofs = nullptr;  // [nl][E]
    double *G = nullptr, *sk = nullptr, *sm = nullptr, *Ye = nullptr, *coords = nullptr;
    double *qp = nullptr, *phi = nullptr, *grad = nullptr;  // rule tables (device)
    std::vector<double> h_phi, h_grad;                       // rule tables (host, kernel parameters)
    int nq = 0;
    int64_t *offs = nullptr;
    int32_t *slots = nullptr;
    uint8_t *ess = nullptr;
    double *xh = nullptr, *yh = nullptr;  // device copies for host-memory calls
    int *d_err = nullptr;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    std::mutex mu;
};

namespace fg {

// tet_rule of crates/element/src/quadrature.rs:259-376: 1 point (order <= 1),
// 4 points (order 2), Grundmann-Moller with s = 2 (order <= 5) or s = 3, the
// per-level weights solved from the x^{2k} moments of the unit tetrahedron.
static void tet_simplex_points(int s, int n, std::vector<std::vector<int>> &out) {
    if (n == 1) {
        out.push_back({s});
        return;
    }
    for (int j0 = 0; j0 <= s; ++j0) {
        std::vector<std::vector<int>> rest;
        tet_simplex_points(s - j0, n - 1, rest);
        for (auto &r : rest) {
            std::vector<int> v{j0};
            v.insert(v.end(), r.begin(), r.end());
            out.push_back(v);
        }
    }
}

static int tet_rule_host(int order, std::vector<double> &pts, std::vector<double> &w) {
    pts.clear();
    w.clear();
    if (order <= 1) {
        pts = {0.25, 0.25, 0.25};
        w = {1.0 / 6.0};
        return 1;
    }
    if (order <= 2) {
        const double a = 0.1381966011250105, b = 0.5854101966249685;
        pts = {a, a, a, b, a, a, a, b, a, a, a, b};
        w.assign(4, 1.0 / 24.0);
        return 4;
    }
    const int s = order <= 5 ? 2 : 3, n = s + 1, d = 3;
    std::vector<std::vector<std::array<double, 3>>> lv(n);
    for (int i = 0; i <= s; ++i) {
        const int si = s - i;
        const double m = 2.0 * si + d + 1;
        std::vector<std::vector<int>> sp;
        tet_simplex_points(si, d + 1, sp);
        for (auto &c : sp) lv[i].push_back({(2.0 * c[1] + 1.0) / m, (2.0 * c[2] + 1.0) / m, (2.0 * c[3] + 1.0) / m});
    }
    auto fact = [](int k) {
        double f = 1.0;
        for (int j = 2; j <= k; ++j) f *= j;
        return f;
    };
    std::vector<std::vector<double>> mat(n, std::vector<double>(n + 1));
    for (int k = 0; k < n; ++k) {
        for (int i = 0; i < n; ++i) {
            double sum = 0.0;
            for (auto &pt : lv[i]) sum += std::pow(pt[0], 2 * k);
            mat[k][i] = sum;
        }
        mat[k][n] = fact(2 * k) / fact(2 * k + 3);
    }
    for (int col = 0; col < n; ++col) {
        int piv = col;
        for (int r = col + 1; r < n; ++r)
            if (std::fabs(mat[r][col]) > std::fabs(mat[piv][col])) piv = r;
        std::swap(mat[col], mat[piv]);
        const double sc = mat[col][col];
        for (int j = col; j <= n; ++j) mat[col][j] /= sc;
        for (int r = 0; r < n; ++r)
            if (r != col) {
                const double f = mat[r][col];
                for (int j = col; j <= n; ++j) mat[r][j] -= f * mat[col][j];
            }
    }
    for (int i = 0; i <= s; ++i)
        for (auto &pt : lv[i]) {
            pts.insert(pts.end(), pt.begin(), pt.end());
            w.push_back(mat[i][n]);
        }
    return (int)w.size();
}

// TetP1 / TetP2 / TetP3 basis values and reference gradients (crates/element/src/lagrange/tet.rs)
static void tet_basis_host(int p, const double *xi, double *phi, double *grad) {
    const double x = xi[0], y = xi[1], z = xi[2];
    const double l1 = 1.0 - x - y - z, l2 = x, l3 = y, l4 = z;
    if (p == 3) {
        // each function is c * f0 f1 f2 with linear factors f = alpha * lambda_i + beta:
        // vertices 1/2 l(3l-1)(3l-2); edge DOFs 9/2 li lj (3li-1) (near i) / (3lj-1) (near j),
        // edges (01, 02, 03, 12, 13, 23); faces 27 li lj lk, faces (012, 013, 023, 123)
        const double L[4] = {l1, l2, l3, l4};
        const double dL[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        struct F { int i; double a, b; };
        F fac[20][3];
        double cc[20];
        for (int v = 0; v < 4; ++v) {
            cc[v] = 0.5;
            fac[v][0] = {v, 1, 0};
            fac[v][1] = {v, 3, -1};
            fac[v][2] = {v, 3, -2};
        }
        const int ed[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
        for (int k = 0; k < 6; ++k)
            for (int h = 0; h < 2; ++h) {
                const int d = 4 + 2 * k + h;
                cc[d] = 4.5;
                fac[d][0] = {ed[k][0], 1, 0};
                fac[d][1] = {ed[k][1], 1, 0};
                fac[d][2] = {h ? ed[k][1] : ed[k][0], 3, -1};
            }
        const int fc[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
        for (int k = 0; k < 4; ++k) {
            cc[16 + k] = 27.0;
            for (int m = 0; m < 3; ++m) fac[16 + k][m] = {fc[k][m], 1, 0};
        }
        for (int d = 0; d < 20; ++d) {
            double f[3];
            for (int m = 0; m < 3; ++m) f[m] = fac[d][m].a * L[fac[d][m].i] + fac[d][m].b;
            phi[d] = cc[d] * f[0] * f[1] * f[2];
            for (int c = 0; c < 3; ++c)
                grad[3 * d + c] = cc[d] * (fac[d][0].a * dL[fac[d][0].i][c] * f[1] * f[2] +
                                           f[0] * fac[d][1].a * dL[fac[d][1].i][c] * f[2] +
                                           f[0] * f[1] * fac[d][2].a * dL[fac[d][2].i][c]);
        }
        return;
    }
    if (p == 1) {
        const double f[4] = {l1, l2, l3, l4};
        const double g[12] = {-1, -1, -1, 1, 0, 0, 0, 1, 0, 0, 0, 1};
        std::copy(f, f + 4, phi);
        std::copy(g, g + 12, grad);
        return;
    }
    const double f[10] = {l1 * (2 * l1 - 1), l2 * (2 * l2 - 1), l3 * (2 * l3 - 1), l4 * (2 * l4 - 1),
                          4 * l1 * l2, 4 * l1 * l3, 4 * l1 * l4, 4 * l2 * l3, 4 * l2 * l4, 4 * l3 * l4};
    const double d0 = 4 * l1 - 1, d1 = 4 * l2 - 1, d2 = 4 * l3 - 1, d3 = 4 * l4 - 1;
    const double g[30] = {-d0, -d0, -d0, d1, 0, 0, 0, d2, 0, 0, 0, d3,
                          4 * (l1 - l2), -4 * l2, -4 * l2, -4 * l3, 4 * (l1 - l3), -4 * l3,
                          -4 * l4, -4 * l4, 4 * (l1 - l4), 4 * l3, 4 * l2, 0, 4 * l4, 0, 4 * l2, 0, 4 * l4, 4 * l3};
    std::copy(f, f + 10, phi);
    std::copy(g, g + 30, grad);
}

static TetArgs tet_args(const fg_tet *t) {
    TetArgs A{};
    A.E = t->E;
    A.N = t->N;
    A.kind = t->kind;
    A.dofs = t->dofs;
    A.G = t->G;
    A.sk = t->sk;
    A.sm = t->sm;
    A.ess = t->ess;
    A.R = TetRule{t->nq, t->phi, t->grad};
    return A;
}

static void tet_free(fg_tet *t) {
    if (!t) return;
    cudaSetDevice(t->device);
    if (t->stream) cudaStreamSynchronize(t->stream);
    void *ptrs[] = {t->dofs, t->G, t->sk, t->sm, t->Ye, t->coords, t->qp, t->phi, t->grad,
                    t->offs, t->slots, t->ess, t->xh, t->yh, t->d_err};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (t->stream && t->own_stream) cudaStreamDestroy(t->stream);
    delete t;
}

template <typename T> static int tet_upload(T **dst, const T *src, size_t n) {
    CK(cudaMalloc(dst, sizeof(T) * std::max<size_t>(n, 1)));
    if (n) CK(cudaMemcpy(*dst, src, sizeof(T) * n, cudaMemcpyDefault));
    FG_LEGACY_FENCE();
    return FG_OK;
}

template <int NL, int MQ>
static void tet_launch_t(fg_tet *t, const TetArgs &A, int eb, const double *x, int constrained, int diag) {
    TetTab<NL, MQ> R{};
    for (int q = 0; q < t->nq; ++q)
        for (int i = 0; i < NL; ++i) {
            R.phi[q][i] = t->h_phi[(size_t)q * NL + i];
            for (int c = 0; c < 3; ++c) R.grad[q][i][c] = t->h_grad[((size_t)q * NL + i) * 3 + c];
        }
    tet_apply_kernel<NL, MQ><<<eb, 128, 0, t->stream>>>(A, R, x, t->Ye, constrained, diag);
}

static int tet_launch_apply(fg_tet *t, const double *x, double *y, int accumulate, int constrained, int diag) {
    const TetArgs A = tet_args(t);
    const int eb = (int)std::min<int64_t>((t->E + 127) / 128, 148 * 16);
    const bool small = t->nq <= 4;
    if (t->p == 1) {
        if (small) tet_launch_t<4, 4>(t, A, eb, x, constrained, diag);
        else tet_launch_t<4, TET_MAXQ>(t, A, eb, x, constrained, diag);
    } else if (t->p == 2) {
        if (small) tet_launch_t<10, 4>(t, A, eb, x, constrained, diag);
        else tet_launch_t<10, TET_MAXQ>(t, A, eb, x, constrained, diag);
    } else {
        if (small) tet_launch_t<20, 4>(t, A, eb, x, constrained, diag);
        else tet_launch_t<20, TET_MAXQ>(t, A, eb, x, constrained, diag);
    }
    const int db = (int)std::min<int64_t>((t->N + 255) / 256, 148 * 16);
    tet_scatter_kernel<<<db, 256, 0, t->stream>>>(A, t->offs, t->slots, t->Ye, diag ? nullptr : x, y, accumulate,
                                                  constrained);
    CK(cudaGetLastError());
    return FG_OK;
}

}  // namespace fg
