// hex_host.cuh -- host side of the unstructured Hex8 operator (fg_op_create_hex):
// validation of the caller's mesh and DOF maps, the element chunks of the
// deterministic scatter, the quadrature-data build and the launches.  Included
// by femgpu.cu after the fg_op handle; an operator built here is an ordinary
// fg_op whose applies and diagonal go through hex_kernels.cuh, so fg_op_apply,
// fg_op_diagonal and fg_pcg serve both mesh kinds.
#pragma once
#include "chunk_plan.h"
#include "hex_kernels.cuh"

// Warps per CTA (a chunk is WARPS * 32 elements), stages of the per-warp
// quadrature-data ring, CTAs per SM the register allocation must allow.
template <int P> struct HexCfg {
    static constexpr int WARPS = P == 3 ? 2 : 4, S = 2, MINB = P == 3 ? 4 : 3;
};
static int hex_chunk_size(int p) {
    return 32 * (p == 1 ? HexCfg<1>::WARPS : p == 2 ? HexCfg<2>::WARPS : HexCfg<3>::WARPS);
}

template <typename T>
static HexApply<T> hex_args(fg_op *op, const T *qd, const T *x, T *y, int accumulate, int constrained,
                            const int *skip) {
    HexApply<T> A{};
    A.E = op->u_E;
    A.N = op->N;
    A.dofs = op->u_dofs;
    A.qd = qd;
    A.ess = op->u_ess;
    A.emsk = op->u_emsk;
    A.x = x;
    A.y = y;
    A.accumulate = accumulate;
    A.constrained = constrained;
    A.skip = skip;
    A.err = op->d_err;
    A.wait_ns = op->wait_ns;
    A.L.cu_off = op->u_cu_off;
    A.L.cu_dof = op->u_cu_dof;
    A.L.cu_pid = op->u_cu_pid;
    A.L.cu_soff = op->u_cu_soff;
    A.L.cu_slots = op->u_cu_slots;
    A.L.part = op->u_part;
    A.L.sh_dof = op->u_sh_dof;
    A.L.sh_off = op->u_sh_off;
    A.L.n_shared = op->u_nshared;
    A.L.max_nu = op->u_max_nu;
    return A;
}

// Raise a kernel's dynamic shared-memory limit to `bytes` on this device (once
// per size reached; set-up calls are serialised by the handle mutexes, and a
// race only repeats the call).
template <typename K> static int hex_smem_limit(K kern, int device, int bytes, std::atomic<int> *lim) {
    if (device < 0 || device >= 64) return fail(FG_CUDA_ERROR, "device id %d out of range", device);
    if (lim[device].load(std::memory_order_acquire) < bytes) {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        lim[device].store(bytes, std::memory_order_release);
    }
    return FG_OK;
}

template <int P, int OPK, typename T>
static int hex_apply_t(fg_op *op, const HexApply<T> &A) {
    constexpr int WARPS = HexCfg<P>::WARPS, S = HexCfg<P>::S, BS = WARPS * 32;
    using SM = HexSmem<P, OPK, T, WARPS, S>;
    auto kern = hex_apply_kernel<P, OPK, T, WARPS, S, HexCfg<P>::MINB>;
    static std::atomic<int> lim[64];
    const int bytes = SM::bytes(op->u_max_nu);
    int rc;
    if ((rc = hex_smem_limit(kern, op->device, bytes, lim))) return rc;
    kern<<<(unsigned)op->u_chunks, BS, bytes, op->stream>>>(A);
    CK(cudaGetLastError());
    return FG_OK;
}

template <typename T> static int hex_shared(fg_op *op, const HexApply<T> &A, int diag) {
    if (!op->u_nshared) return FG_OK;
    const int db = (int)std::min<int64_t>((op->u_nshared + 255) / 256, 148 * 16);
    chunk_shared_kernel<T><<<db, 256, 0, op->stream>>>(A.L, A.ess, A.x, A.y, A.accumulate, A.constrained, diag,
                                                       A.skip);
    CK(cudaGetLastError());
    return FG_OK;
}

// y (+)= A x on native vectors of an unstructured operator (the plain values, then zero pads).
template <typename T>
static int hex_apply(fg_op *op, const T *qd, const T *x, T *y, int accumulate, int constrained, const int *skip) {
    const HexApply<T> A = hex_args<T>(op, qd, x, y, accumulate, constrained, skip);
    int rc;
    switch (op->p * 4 + op->kind) {
    case 1 * 4 + 1: rc = hex_apply_t<1, 1, T>(op, A); break;
    case 1 * 4 + 2: rc = hex_apply_t<1, 2, T>(op, A); break;
    case 1 * 4 + 3: rc = hex_apply_t<1, 3, T>(op, A); break;
    case 2 * 4 + 1: rc = hex_apply_t<2, 1, T>(op, A); break;
    case 2 * 4 + 2: rc = hex_apply_t<2, 2, T>(op, A); break;
    case 2 * 4 + 3: rc = hex_apply_t<2, 3, T>(op, A); break;
    case 3 * 4 + 1: rc = hex_apply_t<3, 1, T>(op, A); break;
    case 3 * 4 + 2: rc = hex_apply_t<3, 2, T>(op, A); break;
    default: rc = hex_apply_t<3, 3, T>(op, A); break;
    }
    return rc ? rc : hex_shared<T>(op, A, 0);
}

template <int P, int OPK> static int hex_diag_t(fg_op *op, const HexApply<double> &A) {
    constexpr int BS = HexCfg<P>::WARPS * 32, NL = (P + 1) * (P + 1) * (P + 1);
    auto kern = hex_diag_kernel<P, OPK, BS>;
    static std::atomic<int> lim[64];
    const int bytes = (int)(sizeof(double) * NL * BS + chunk_list_smem(NL, BS, op->u_max_nu));
    int rc;
    if ((rc = hex_smem_limit(kern, op->device, bytes, lim))) return rc;
    kern<<<(unsigned)op->u_chunks, BS, bytes, op->stream>>>(A);
    CK(cudaGetLastError());
    return FG_OK;
}

static int hex_diag(fg_op *op, double *y, int constrained) {
    const HexApply<double> A = hex_args<double>(op, op->qd, nullptr, y, 0, constrained, nullptr);
    int rc;
    switch (op->p * 4 + op->kind) {
    case 1 * 4 + 1: rc = hex_diag_t<1, 1>(op, A); break;
    case 1 * 4 + 2: rc = hex_diag_t<1, 2>(op, A); break;
    case 1 * 4 + 3: rc = hex_diag_t<1, 3>(op, A); break;
    case 2 * 4 + 1: rc = hex_diag_t<2, 1>(op, A); break;
    case 2 * 4 + 2: rc = hex_diag_t<2, 2>(op, A); break;
    case 2 * 4 + 3: rc = hex_diag_t<2, 3>(op, A); break;
    case 3 * 4 + 1: rc = hex_diag_t<3, 1>(op, A); break;
    case 3 * 4 + 2: rc = hex_diag_t<3, 2>(op, A); break;
    default: rc = hex_diag_t<3, 3>(op, A); break;
    }
    return rc ? rc : hex_shared<double>(op, A, 1);
}

template <int P, int OPK> static void hex_setup_launch(fg_op *op, const HexSetup &S) {
    const int64_t total = S.E * (P + 1) * (P + 1) * (P + 1);
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
    hex_setup_kernel<P, OPK, double><<<blocks, 256, 0, op->stream>>>(S, op->qd);
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
    // elements in the Morton order of their vertex centroids, padded to whole
    // 32-element groups (padding: eid -1, map -1), cut into chunks of the CTA size
    const int CE = hex_chunk_size(order);
    if (nl * CE > 65536) return fail(FG_UNSUPPORTED, "chunk of %d elements too large for 16-bit slots", CE);
    std::vector<int32_t> perm;
    {
        std::vector<double> h_xyz((size_t)n_nodes * 3);
        CK(cudaMemcpy(h_xyz.data(), coords, sizeof(double) * h_xyz.size(), cudaMemcpyDefault));
        std::vector<double> cen((size_t)E * 3);
        for (int64_t e = 0; e < E; ++e)
            for (int a = 0; a < 3; ++a) {
                double sum = 0.0;
                for (int v = 0; v < 8; ++v) sum += h_xyz[3 * (size_t)h_conn[(size_t)e * 8 + v] + a];
                cen[3 * (size_t)e + a] = 0.125 * sum;
            }
        morton_order(cen, E, perm);
    }
    const int64_t Ep = (E + 31) / 32 * 32;
    std::vector<int32_t> eid((size_t)Ep, -1), smap((size_t)Ep * nl, -1), sdofs((size_t)Ep * nl, -1);
    for (int64_t s = 0; s < E; ++s) {
        eid[(size_t)s] = perm[(size_t)s];
        for (int k = 0; k < nl; ++k) {
            const int32_t d = lexmap[(size_t)perm[(size_t)s] * nl + k];
            smap[(size_t)s * nl + k] = d;
            sdofs[(size_t)k * Ep + s] = d;
        }
    }
    ChunkPlan plan;
    plan_chunk_lists(smap, Ep, N, nl, CE, plan);
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
    op->u_chunks = plan.n_chunks;
    op->u_nshared = (int64_t)plan.sh_dof.size();
    op->u_max_nu = plan.max_nu;
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
    {
        auto up = [](auto **dst, const auto &v) {
            using V = typename std::remove_reference<decltype(v)>::type::value_type;
            const size_t n = std::max<size_t>(v.size(), 1);
            if (cudaMalloc(dst, sizeof(V) * n) != cudaSuccess) return false;
            return v.empty() || cudaMemcpy(*dst, v.data(), sizeof(V) * v.size(), cudaMemcpyHostToDevice) == cudaSuccess;
        };
        std::vector<uint64_t> em((size_t)Ep, 0ull);
        for (int64_t s = 0; s < Ep; ++s)
            for (int k = 0; k < nl; ++k) {
                const int32_t d = smap[(size_t)s * nl + k];
                if (d >= 0 && mask[(size_t)d]) em[(size_t)s] |= 1ull << k;
            }
        if (!up(&op->u_emsk, em) || !up(&op->u_cu_off, plan.cu_off) || !up(&op->u_cu_dof, plan.cu_dof) || !up(&op->u_cu_pid, plan.cu_pid) ||
            !up(&op->u_cu_soff, plan.cu_soff) || !up(&op->u_cu_slots, plan.cu_slots) ||
            !up(&op->u_sh_dof, plan.sh_dof) || !up(&op->u_sh_off, plan.sh_off) ||
            cudaMalloc(&op->u_part, sizeof(double) * std::max<int64_t>(plan.n_part, 1)) != cudaSuccess)
            return bail(fail(FG_CUDA_ERROR, "upload of the chunk lists failed"));
    }

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

extern "C" FG_API int64_t fg_op_chunks(const fg_op *op) {
    if (!op) return fail(FG_INVALID_ARGUMENT, "NULL op");
    return op->unstr ? op->u_chunks : 0;
}
