// hex_host.cuh -- host side of the unstructured Hex8 operator (fg_op_create_hex):
// validation of the caller's mesh and DOF maps, the element colouring of the
// deterministic scatter, the quadrature-data build and the launches.  Included
// by femgpu.cu after the fg_op handle; an operator built here is an ordinary
// fg_op whose applies and diagonal go through hex_kernels.cuh, so fg_op_apply,
// fg_op_diagonal and fg_pcg serve both mesh kinds.
#pragma once
#include "hex_kernels.cuh"

// Warps per CTA, stages of the per-warp quadrature-data ring, CTAs per SM
// the register allocation must allow (shared memory allows 5 at Q2 FP64).
template <int P> struct HexCfg { static constexpr int WARPS = 2, S = P == 3 ? 2 : 3, MINB = P == 3 ? 4 : 5; };

template <typename T>
static HexApply<T> hex_args(fg_op *op, const T *qd, const T *x, T *y, int constrained, const int *skip) {
    HexApply<T> A{};
    A.E = op->u_E;
    A.N = op->N;
    A.dofs = op->u_dofs;
    A.qd = qd;
    A.ess = op->u_ess;
    A.x = x;
    A.y = y;
    A.constrained = constrained;
    A.skip = skip;
    A.err = op->d_err;
    A.wait_ns = op->wait_ns;
    return A;
}

template <int P, int OPK, typename T>
static int hex_apply_t(fg_op *op, HexApply<T> A) {
    constexpr int WARPS = HexCfg<P>::WARPS, S = HexCfg<P>::S, BS = WARPS * 32;
    using SM = HexSmem<P, OPK, T, WARPS, S>;
    auto kern = hex_apply_kernel<P, OPK, T, WARPS, S, HexCfg<P>::MINB>;
    static std::atomic<bool> attr_set[64];  // per device, set once
    if (op->device < 0 || op->device >= 64) return fail(FG_CUDA_ERROR, "device id %d out of range", op->device);
    if (!attr_set[op->device].load(std::memory_order_acquire)) {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SM::bytes));
        attr_set[op->device].store(true, std::memory_order_release);
    }
    for (size_t c = 0; c + 1 < op->u_col.size(); ++c) {
        A.e0 = op->u_col[c];
        A.e1 = op->u_col[c + 1];
        const int64_t n = A.e1 - A.e0;  // a multiple of 32
        if (n <= 0) continue;
        kern<<<(unsigned)((n + BS - 1) / BS), BS, SM::bytes, op->stream>>>(A);
        CK(cudaGetLastError());
    }
    return FG_OK;
}

// y (+)= A x on native vectors of an unstructured operator (the plain values, then zero pads).
template <typename T>
static int hex_apply(fg_op *op, const T *qd, const T *x, T *y, int accumulate, int constrained, const int *skip) {
    HexApply<T> A = hex_args<T>(op, qd, x, y, constrained, skip);
    hex_init_kernel<T><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(A, accumulate);
    CK(cudaGetLastError());
    switch (op->p * 4 + op->kind) {
    case 1 * 4 + 1: return hex_apply_t<1, 1, T>(op, A);
    case 1 * 4 + 2: return hex_apply_t<1, 2, T>(op, A);
    case 1 * 4 + 3: return hex_apply_t<1, 3, T>(op, A);
    case 2 * 4 + 1: return hex_apply_t<2, 1, T>(op, A);
    case 2 * 4 + 2: return hex_apply_t<2, 2, T>(op, A);
    case 2 * 4 + 3: return hex_apply_t<2, 3, T>(op, A);
    case 3 * 4 + 1: return hex_apply_t<3, 1, T>(op, A);
    case 3 * 4 + 2: return hex_apply_t<3, 2, T>(op, A);
    default: return hex_apply_t<3, 3, T>(op, A);
    }
}

template <int P, int OPK> static int hex_diag_t(fg_op *op, HexApply<double> A) {
    for (size_t c = 0; c + 1 < op->u_col.size(); ++c) {
        A.e0 = op->u_col[c];
        A.e1 = op->u_col[c + 1];
        const int64_t n = A.e1 - A.e0;
        if (n <= 0) continue;
        hex_diag_kernel<P, OPK><<<(unsigned)((n + 127) / 128), 128, 0, op->stream>>>(A);
        CK(cudaGetLastError());
    }
    return FG_OK;
}

static int hex_diag(fg_op *op, double *y, int constrained) {
    HexApply<double> A = hex_args<double>(op, op->qd, nullptr, y, constrained, nullptr);
    hex_init_kernel<double><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(A, 0);
    CK(cudaGetLastError());
    switch (op->p * 4 + op->kind) {
    case 1 * 4 + 1: return hex_diag_t<1, 1>(op, A);
    case 1 * 4 + 2: return hex_diag_t<1, 2>(op, A);
    case 1 * 4 + 3: return hex_diag_t<1, 3>(op, A);
    case 2 * 4 + 1: return hex_diag_t<2, 1>(op, A);
    case 2 * 4 + 2: return hex_diag_t<2, 2>(op, A);
    case 2 * 4 + 3: return hex_diag_t<2, 3>(op, A);
    case 3 * 4 + 1: return hex_diag_t<3, 1>(op, A);
    case 3 * 4 + 2: return hex_diag_t<3, 2>(op, A);
    default: return hex_diag_t<3, 3>(op, A);
    }
}

template <int P, int OPK> static void hex_setup_launch(fg_op *op, const HexSetup &S) {
    const int64_t total = S.E * (P + 1) * (P + 1) * (P + 1);
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
    hex_setup_kernel<P, OPK, double><<<blocks, 256, 0, op->stream>>>(S, op->qd);
}

// Greedy element colouring: no two elements of a colour share a DOF.  Per DOF
// a 64-bit mask of the colours of the elements already placed on it; each
// element takes the lowest colour none of its DOFs has.  Returns the number of
// colours, or -1 if an element would need a 65th.
static int hex_colour(int64_t E, int nl, int64_t N, const std::vector<int32_t> &ed, std::vector<uint8_t> &col) {
    std::vector<uint64_t> used((size_t)N, 0);
    col.assign((size_t)E, 0);
    int ncol = 0;
    for (int64_t e = 0; e < E; ++e) {
        uint64_t forb = 0;
        for (int k = 0; k < nl; ++k) forb |= used[(size_t)ed[(size_t)e * nl + k]];
        if (forb == ~0ull) return -1;
        int c = 0;
        while (forb >> c & 1ull) ++c;
        col[(size_t)e] = (uint8_t)c;
        ncol = std::max(ncol, c + 1);
        for (int k = 0; k < nl; ++k) used[(size_t)ed[(size_t)e * nl + k]] |= 1ull << c;
    }
    return ncol;
}

extern "C" FG_API int fg_op_create_hex(int order, int64_t n_nodes, const double *coords, int64_t n_elem,
                                       const uint32_t *conn, const uint32_t *elem_dofs, int64_t n_dofs, int kind,
                                       double c_mass, double c_diff, const double *kappa_q, double kappa_const,
                                       const double *rho_q, double rho_const, const uint32_t *ess_dofs,
                                       int64_t n_ess, fg_op **out) {
    t_last_status = FG_OK;
    if (!out) return fail(FG_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (order < 1 || order > FG_MAXP)
        return fail(FG_UNSUPPORTED, "unsupported order %d (supported: 1..%d)", order, FG_MAXP);
    if (kind < 1 || kind > 3) return fail(FG_INVALID_ARGUMENT, "bad operator kind %d", kind);
    if (n_nodes < 8 || n_elem < 1 || n_dofs < 1 || !coords || !conn)
        return fail(FG_INVALID_ARGUMENT, "empty mesh or NULL coordinates / connectivity");
    if (order > 1 && !elem_dofs) return fail(FG_INVALID_ARGUMENT, "order %d needs the element DOF maps", order);
    if (n_ess < 0 || (n_ess > 0 && !ess_dofs)) return fail(FG_INVALID_ARGUMENT, "bad essential-DOF list");
    if (n_dofs >= ((int64_t)1 << 31) - 4 || n_elem >= ((int64_t)1 << 31))
        return fail(FG_INVALID_ARGUMENT, "more than 2^31 DOFs or elements");
    const int D = order + 1, nl = D * D * D, Q3 = nl;
    const int64_t E = n_elem, N = n_dofs;

    // caller's maps to the host (host or device pointers; cudaMemcpyDefault handles both)
    std::vector<uint32_t> h_conn((size_t)E * 8), h_map;
    CK(cudaMemcpy(h_conn.data(), conn, sizeof(uint32_t) * h_conn.size(), cudaMemcpyDefault));
    if (elem_dofs) {
        h_map.resize((size_t)E * nl);
        CK(cudaMemcpy(h_map.data(), elem_dofs, sizeof(uint32_t) * h_map.size(), cudaMemcpyDefault));
    } else {
        h_map = h_conn;  // order 1: DOF = node (DofManager::build_p1, dof_manager.rs:137-160)
    }
    for (uint32_t v : h_conn)
        if ((int64_t)v >= n_nodes) return fail(FG_BOUNDS, "connectivity names node %u of %lld", v, (long long)n_nodes);
    for (uint32_t d : h_map)
        if ((int64_t)d >= N) return fail(FG_BOUNDS, "element DOF map names DOF %u of %lld", d, (long long)N);
    // local order -> tensor order (c, b, a): order 1 takes the HexQ1 vertex
    // order (crates/element/src/lagrange/hex.rs:27-36), orders 2-3 the tensor
    // order itself
    std::vector<int32_t> lexmap((size_t)E * nl);
    for (int64_t e = 0; e < E; ++e)
        for (int c = 0; c < D; ++c)
            for (int b = 0; b < D; ++b)
                for (int a = 0; a < D; ++a) {
                    const int k = (c * D + b) * D + a;
                    const int src = order == 1 ? (b ? (a ? 2 : 3) : (a ? 1 : 0)) + 4 * c : k;
                    lexmap[(size_t)e * nl + k] = (int32_t)h_map[(size_t)e * nl + src];
                }
    std::vector<uint8_t> colour;
    const int ncol = hex_colour(E, nl, N, lexmap, colour);
    if (ncol < 0) return fail(FG_UNSUPPORTED, "element colouring needs more than 64 colours");
    // elements sorted by colour (stable: the caller's order within a colour),
    // each colour padded to whole 32-element chunks (padding: eid -1, map -1)
    std::vector<int64_t> count((size_t)ncol, 0), start((size_t)ncol + 1, 0);
    for (uint8_t c : colour) ++count[c];
    for (int c = 0; c < ncol; ++c) start[(size_t)c + 1] = start[(size_t)c] + (count[(size_t)c] + 31) / 32 * 32;
    const int64_t Ep = start[(size_t)ncol];
    if (Ep >= ((int64_t)1 << 31)) return fail(FG_INVALID_ARGUMENT, "more than 2^31 padded elements");
    std::vector<int32_t> eid((size_t)Ep, -1), sdofs((size_t)Ep * nl, -1);
    {
        std::vector<int64_t> pos(start.begin(), start.end() - 1);
        for (int64_t e = 0; e < E; ++e) eid[(size_t)pos[colour[(size_t)e]]++] = (int32_t)e;
    }
    for (int k = 0; k < nl; ++k)
        for (int64_t s = 0; s < Ep; ++s)
            if (eid[(size_t)s] >= 0) sdofs[(size_t)k * Ep + s] = lexmap[(size_t)eid[(size_t)s] * nl + k];
    std::vector<uint8_t> mask((size_t)N, 0);
    if (n_ess > 0) {
        std::vector<uint32_t> h_ess((size_t)n_ess);
        CK(cudaMemcpy(h_ess.data(), ess_dofs, sizeof(uint32_t) * h_ess.size(), cudaMemcpyDefault));
        for (uint32_t d : h_ess) {
            if ((int64_t)d >= N) return fail(FG_BOUNDS, "essential DOF %u of %lld", d, (long long)N);
            mask[d] = 1;
        }
    }

    int dev = 0;
    CK(cudaGetDevice(&dev));
    int rc = ensure_tables(dev);
    if (rc) return rc;
    fg_op *op = new fg_op();
    op->device = dev;
    op->kind = kind;
    op->p = order;
    op->unstr = true;
    op->u_E = Ep;
    op->u_col = start;
    op->N = N;
    // native vectors: one row of the N plain values padded with zeros to a
    // multiple of 4 (the solver's vector kernels work in 4-wide groups); no tiles
    op->Nn = round_up((int)N, 4);
    Grid &g = op->g;
    g.p = order;
    g.NI = (int)N;
    g.NJ = g.NK = 1;
    g.NIp = (int)op->Nn;
    g.WY = 1;
    g.TZ = 1;
    auto bail = [&](int s) { free_op(op); return s; };
    if (cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(FG_CUDA_ERROR, "cudaStreamCreate failed"));
    op->own_stream = true;
    {
        const char *e = std::getenv("FG_SOLVER_GRAPHS");
        op->graphs = !(e && e[0] == '0');
        const char *fp = std::getenv("FG_FUSED_PCG");
        op->fused_pcg = !(fp && fp[0] == '0');
    }
    if (cudaMalloc(&op->d_err, sizeof(int)) != cudaSuccess || cudaMemset(op->d_err, 0, sizeof(int)) ||
        cudaMalloc(&op->st, sizeof(SolverState)) != cudaSuccess ||
        cudaMemset(op->st, 0, sizeof(SolverState)) != cudaSuccess)
        return bail(fail(FG_CUDA_ERROR, "cudaMalloc failed"));
    if ((rc = alloc_vec(&op->xs, op->Nn)) || (rc = alloc_vec(&op->ys, op->Nn)) || (rc = alloc_vec(&op->face, 1)) ||
        (rc = alloc_vec(&op->partials, VEC_GRID * 4)))
        return bail(rc);
    cudaEventCreate(&op->ev0);
    cudaEventCreate(&op->ev1);
    if (cudaMalloc(&op->u_dofs, sizeof(int32_t) * sdofs.size()) ||
        cudaMemcpy(op->u_dofs, sdofs.data(), sizeof(int32_t) * sdofs.size(), cudaMemcpyHostToDevice) ||
        cudaMalloc(&op->u_ess, (size_t)N) || cudaMemcpy(op->u_ess, mask.data(), (size_t)N, cudaMemcpyHostToDevice))
        return bail(fail(FG_CUDA_ERROR, "upload of the element maps failed"));

    // quadrature data
    const int NC = kind == FG_MASS ? 1 : (kind == FG_DIFF ? 6 : 7);
    op->qsize = Ep * Q3 * NC;
    if ((rc = alloc_vec(&op->qd, op->qsize))) return bail(rc);
    int32_t *d_eid = nullptr;
    uint32_t *d_conn = nullptr;
    double *d_xyz = nullptr, *d_kq = nullptr, *d_rq = nullptr;
    auto cleanup_in = [&]() {
        if (d_eid) cudaFree(d_eid);
        if (d_conn) cudaFree(d_conn);
        if (d_xyz) cudaFree(d_xyz);
        if (d_kq) cudaFree(d_kq);
        if (d_rq) cudaFree(d_rq);
    };
    bool up_ok = !cudaMalloc(&d_eid, sizeof(int32_t) * Ep) &&
                 !cudaMemcpy(d_eid, eid.data(), sizeof(int32_t) * Ep, cudaMemcpyHostToDevice) &&
                 !cudaMalloc(&d_conn, sizeof(uint32_t) * E * 8) &&
                 !cudaMemcpy(d_conn, h_conn.data(), sizeof(uint32_t) * E * 8, cudaMemcpyHostToDevice) &&
                 !cudaMalloc(&d_xyz, sizeof(double) * 3 * n_nodes) &&
                 !cudaMemcpy(d_xyz, coords, sizeof(double) * 3 * n_nodes, cudaMemcpyDefault);
    if (up_ok && kappa_q)
        up_ok = !cudaMalloc(&d_kq, sizeof(double) * E * Q3) &&
                !cudaMemcpy(d_kq, kappa_q, sizeof(double) * E * Q3, cudaMemcpyDefault);
    if (up_ok && rho_q)
        up_ok = !cudaMalloc(&d_rq, sizeof(double) * E * Q3) &&
                !cudaMemcpy(d_rq, rho_q, sizeof(double) * E * Q3, cudaMemcpyDefault);
    if (!up_ok || cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess) {
        cleanup_in();
        return bail(fail(FG_CUDA_ERROR, "upload of the mesh and coefficients failed"));
    }
    HexSetup S{};
    S.E = Ep;
    S.eid = d_eid;
    S.conn = d_conn;
    S.coords = d_xyz;
    S.kappa_q = d_kq;
    S.rho_q = d_rq;
    S.kappa_c = kappa_const;
    S.rho_c = rho_const;
    S.c_m = c_mass;
    S.c_k = c_diff;
    gauss_legendre(order + 1, S.gx, S.gw);
    S.err = op->d_err;
    switch (order * 4 + kind) {
    case 1 * 4 + 1: hex_setup_launch<1, 1>(op, S); break;
    case 1 * 4 + 2: hex_setup_launch<1, 2>(op, S); break;
    case 1 * 4 + 3: hex_setup_launch<1, 3>(op, S); break;
    case 2 * 4 + 1: hex_setup_launch<2, 1>(op, S); break;
    case 2 * 4 + 2: hex_setup_launch<2, 2>(op, S); break;
    case 2 * 4 + 3: hex_setup_launch<2, 3>(op, S); break;
    case 3 * 4 + 1: hex_setup_launch<3, 1>(op, S); break;
    case 3 * 4 + 2: hex_setup_launch<3, 2>(op, S); break;
    default: hex_setup_launch<3, 3>(op, S); break;
    }
    const cudaError_t le = cudaGetLastError();
    const cudaError_t se = cudaStreamSynchronize(op->stream);
    cleanup_in();
    if (le != cudaSuccess || se != cudaSuccess)
        return bail(fail(FG_CUDA_ERROR, "quadrature-data setup failed: %s",
                         cudaGetErrorString(le != cudaSuccess ? le : se)));
    int herr = 0;
    if (cudaMemcpy(&herr, op->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return bail(fail(FG_CUDA_ERROR, "reading the set-up error word failed"));
    if (herr & FG_DERR_BOUNDS) return bail(fail(FG_BOUNDS, "degenerate element (det J = 0)"));
    *out = op;
    return FG_OK;
}

extern "C" FG_API int fg_op_colours(const fg_op *op) {
    if (!op) return fail(FG_INVALID_ARGUMENT, "NULL op");
    return op->unstr ? (int)op->u_col.size() - 1 : 0;
}
