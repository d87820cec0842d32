// tet_host.cuh -- host side of the tetrahedral PA operator (included by
// femgpu.cu, single translation unit).
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <mutex>
#include <vector>

#include "chunk_plan.h"
#include "tet_kernels.cuh"

struct fg_tet {
    int device = 0;
    int p = 1, nl = 4, kind = 2;
    int64_t E = 0, N = 0, n_nodes = 0;
    int32_t *dofs = nullptr;  // [nl][E] caller's element order (setup, quadrature points)
    double *G = nullptr, *sk = nullptr, *sm = nullptr, *Sm = nullptr, *coords = nullptr;  // chunk order
    double *qp = nullptr, *phi = nullptr, *grad = nullptr;  // rule tables (device)
    std::vector<double> h_phi, h_grad;                       // rule tables (host, kernel parameters)
    int nq = 0;
    // chunked scatter
    int CE = 0, max_nu = 0, n_chunks = 0, wide = 0;  // wide: 512-thread CTAs for the P2 moment form
    int64_t n_shared = 0, n_part = 0;
    int32_t *edof = nullptr;   // [nl][E] chunk order
    uint32_t *emsk = nullptr;  // [E] chunk order
    uint16_t *cu_slots = nullptr;
    int32_t *cu_off = nullptr, *cu_dof = nullptr, *cu_pid = nullptr, *cu_soff = nullptr;
    int32_t *sh_dof = nullptr, *sh_off = nullptr;
    double *part = nullptr;
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

static TetChunk tet_chunk_args(const fg_tet *t) {
    TetChunk C{};
    C.E = t->E;
    C.N = t->N;
    C.CE = t->CE;
    C.G = t->G;
    C.Sm = t->Sm;
    C.sk = t->sk;
    C.sm = t->sm;
    C.edof = t->edof;
    C.emsk = t->emsk;
    C.ess = t->ess;
    C.L.cu_off = t->cu_off;
    C.L.cu_dof = t->cu_dof;
    C.L.cu_pid = t->cu_pid;
    C.L.cu_soff = t->cu_soff;
    C.L.cu_slots = t->cu_slots;
    C.L.part = t->part;
    C.L.sh_dof = t->sh_dof;
    C.L.sh_off = t->sh_off;
    C.L.n_shared = t->n_shared;
    C.L.max_nu = t->max_nu;
    return C;
}

static void tet_free(fg_tet *t) {
    if (!t) return;
    cudaSetDevice(t->device);
    if (t->stream) cudaStreamSynchronize(t->stream);
    void *ptrs[] = {t->dofs, t->G, t->sk, t->sm, t->Sm, t->coords, t->qp, t->phi, t->grad, t->edof, t->emsk, t->cu_slots,
                    t->cu_off, t->cu_dof, t->cu_pid, t->cu_soff, t->sh_dof, t->sh_off, t->part, t->ess, t->xh,
                    t->yh, t->d_err};
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

// Element order (Morton order of the centroids of the four vertex nodes, the
// first four local DOFs) and the chunk DOF lists.  h = element map [E][nl] in
// the caller's order; perm[n] = the caller's element at position n.
static void tet_plan_chunks(const std::vector<int32_t> &h, const std::vector<double> &coords, int64_t E,
                            int64_t N, int nl, int CE, std::vector<int32_t> &perm, ChunkPlan &P) {
    std::vector<double> cen((size_t)E * 3);
    for (int64_t e = 0; e < E; ++e)
        for (int a = 0; a < 3; ++a) {
            double s = 0.0;
            for (int v = 0; v < 4; ++v) s += coords[3 * (size_t)h[e * nl + v] + a];
            cen[3 * e + a] = 0.25 * s;
        }
    morton_order(cen, E, perm);
    std::vector<int32_t> smap((size_t)E * nl);
    for (int64_t n = 0; n < E; ++n)
        for (int i = 0; i < nl; ++i) smap[(size_t)n * nl + i] = h[(size_t)perm[n] * nl + i];
    plan_chunk_lists(smap, E, N, nl, CE, P);
}

template <int NL, int MQ, bool MOM, int BT>
static int tet_launch_t(fg_tet *t, const TetChunk &C, const double *x, double *y, int accumulate, int constrained,
                        int diag) {
    TetTab<NL, MQ> R{};
    if (!MOM)
        for (int q = 0; q < t->nq; ++q)
            for (int i = 0; i < NL; ++i) {
                R.phi[q][i] = t->h_phi[(size_t)q * NL + i];
                for (int c = 0; c < 3; ++c) R.grad[q][i][c] = t->h_grad[((size_t)q * NL + i) * 3 + c];
            }
    const size_t smem = tet_chunk_smem(NL, t->CE, t->max_nu);
    if (smem > 48 * 1024)
        CK(cudaFuncSetAttribute(tet_chunk_kernel<NL, MQ, MOM, BT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
    tet_chunk_kernel<NL, MQ, MOM, BT><<<t->n_chunks, BT, smem, t->stream>>>(C, t->kind, t->nq, R, x, y, accumulate,
                                                                            constrained, diag);
    return FG_OK;
}

static int tet_launch_apply(fg_tet *t, const double *x, double *y, int accumulate, int constrained, int diag) {
    const TetChunk C = tet_chunk_args(t);
    const bool small = t->nq <= 4;
    const bool mom = !diag && t->kind == 2 && t->p <= 2;
    int rc;
    if (t->p == 1) {
        if (mom) rc = tet_launch_t<4, 1, true, 256>(t, C, x, y, accumulate, constrained, diag);
        else if (small) rc = tet_launch_t<4, 4, false, 256>(t, C, x, y, accumulate, constrained, diag);
        else rc = tet_launch_t<4, TET_MAXQ, false, 256>(t, C, x, y, accumulate, constrained, diag);
    } else if (t->p == 2) {
        if (mom && t->wide) rc = tet_launch_t<10, 1, true, 512>(t, C, x, y, accumulate, constrained, diag);
        else if (mom) rc = tet_launch_t<10, 1, true, 256>(t, C, x, y, accumulate, constrained, diag);
        else if (small) rc = tet_launch_t<10, 4, false, 256>(t, C, x, y, accumulate, constrained, diag);
        else rc = tet_launch_t<10, TET_MAXQ, false, 256>(t, C, x, y, accumulate, constrained, diag);
    } else {
        if (small) rc = tet_launch_t<20, 4, false, 256>(t, C, x, y, accumulate, constrained, diag);
        else rc = tet_launch_t<20, TET_MAXQ, false, 256>(t, C, x, y, accumulate, constrained, diag);
    }
    if (rc) return rc;
    if (t->n_shared) {
        const int db = (int)std::min<int64_t>((t->n_shared + 255) / 256, 148 * 16);
        chunk_shared_kernel<double><<<db, 256, 0, t->stream>>>(C.L, t->ess, diag ? nullptr : x, y, accumulate,
                                                               constrained, diag, nullptr);
    }
    CK(cudaGetLastError());
    return FG_OK;
}

}  // namespace fg
