// femgpu.cu -- host side of libfemgpu.so: the C ABI of include/femgpu.h over
// the sm_100a kernels of pa_kernels.cuh and vec_kernels.cuh.
//
// There is no CPU fallback: every numeric entry point runs on the GPU and
// fails with FG_CUDA_ERROR when no usable device is present.
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <functional>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/femgpu.h"
#include "fg_common.cuh"
#include "pa_kernels.cuh"
#include "vec_kernels.cuh"
#include "form_kernels.cuh"


using namespace fg;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local int t_last_status = FG_OK;
static thread_local std::string t_last_msg;

static int fail(int status, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_last_status = status;
    t_last_msg = buf;
    return status;
}
#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(FG_CUDA_ERROR, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                               \
    } while (0)
// cudaMemset, cudaMemcpy from pageable host memory and launches without a
// stream go to the legacy default stream, which the library's non-blocking
// streams (and the caller's) do not wait for, and the first two can still be
// running when the call returns.  Set-up paths call this before any launch on
// another stream reads what they wrote.
#define FG_LEGACY_FENCE() CK(cudaStreamSynchronize(cudaStreamLegacy))
// Entry points built on the structured box (its DOF lattice, item tiles or
// compressed qdata) refuse operators of an unstructured Hex8 mesh.
#define FG_NEED_BOX(op, what)                                                                  \
    do {                                                                                       \
        if ((op) && (op)->unstr)                                                               \
            return fail(FG_UNSUPPORTED, "%s needs a structured hex box (fg_op_create)", what); \
    } while (0)

#include "unet_host.cuh"
#include "tet_host.cuh"

// ---------------------------------------------------------------------------
// 1-D tables: Gauss-Legendre (crates/element/src/quadrature.rs:12-32) and
// equispaced Lagrange polynomials (quad.rs:92-105, seg.rs:119-121 conventions).
// ---------------------------------------------------------------------------
static void gauss_legendre(int n, double *x, double *w) {
    switch (n) {
    case 1: x[0] = 0.0; w[0] = 2.0; break;
    case 2: { double a = 1.0 / std::sqrt(3.0); x[0] = -a; x[1] = a; w[0] = w[1] = 1.0; } break;
    case 3: {
        double a = std::sqrt(3.0 / 5.0);
        x[0] = -a; x[1] = 0.0; x[2] = a;
        w[0] = 5.0 / 9.0; w[1] = 8.0 / 9.0; w[2] = 5.0 / 9.0;
    } break;
    default: {
        double a = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
        double b = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
        double wa = (18.0 + std::sqrt(30.0)) / 36.0, wb = (18.0 - std::sqrt(30.0)) / 36.0;
        x[0] = -b; x[1] = -a; x[2] = a; x[3] = b;
        w[0] = wb; w[1] = wa; w[2] = wa; w[3] = wb;
    } break;
    }
}

static void lagrange1d(int p, double xi, double *phi, double *dphi) {
    double nodes[FG_MAXP + 1];
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

static std::mutex g_init_mu;
static bool g_tables_ready[64];

static int ensure_tables(int dev) {
    std::lock_guard<std::mutex> lk(g_init_mu);
    if (dev < 0 || dev >= 64) return fail(FG_CUDA_ERROR, "device id %d out of range", dev);
    if (g_tables_ready[dev]) return FG_OK;
    double B[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1] = {}, G[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1] = {};
    float Bf[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1] = {}, Gf[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1] = {};
    for (int p = 1; p <= FG_MAXP; ++p) {
        double x[4], w[4];
        gauss_legendre(p + 1, x, w);
        for (int q = 0; q <= p; ++q) {
            double phi[4], dphi[4];
            lagrange1d(p, x[q], phi, dphi);
            for (int d = 0; d <= p; ++d) {
                B[p - 1][q][d] = phi[d];
                G[p - 1][q][d] = dphi[d];
                Bf[p - 1][q][d] = (float)phi[d];
                Gf[p - 1][q][d] = (float)dphi[d];
            }
        }
    }
    CK(cudaMemcpyToSymbol(c_B64, B, sizeof B));
    CK(cudaMemcpyToSymbol(c_G64, G, sizeof G));
    CK(cudaMemcpyToSymbol(c_B32, Bf, sizeof Bf));
    CK(cudaMemcpyToSymbol(c_G32, Gf, sizeof Gf));
    float2 GB[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1] = {}, BG[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1] = {},
           BB[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1] = {};
    for (int p = 0; p < FG_MAXP; ++p)
        for (int q = 0; q <= FG_MAXP; ++q)
            for (int d = 0; d <= FG_MAXP; ++d) {
                GB[p][q][d] = make_float2(Gf[p][q][d], Bf[p][q][d]);
                BG[p][q][d] = make_float2(Bf[p][q][d], Gf[p][q][d]);
                BB[p][q][d] = make_float2(Bf[p][q][d], Bf[p][q][d]);
            }
    CK(cudaMemcpyToSymbol(c_GB32, GB, sizeof GB));
    CK(cudaMemcpyToSymbol(c_BG32, BG, sizeof BG));
    CK(cudaMemcpyToSymbol(c_BB32, BB, sizeof BB));
    // Dq = G B^-1 per order (B inverted by Gauss-Jordan with partial pivoting, in FP64)
    float DQ[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1] = {};
    double DQd[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1] = {};
    for (int p = 1; p <= FG_MAXP; ++p) {
        const int n = p + 1;
        double a[4][8] = {};
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                a[i][j] = B[p - 1][i][j];
                a[i][n + j] = i == j ? 1.0 : 0.0;
            }
        for (int c = 0; c < n; ++c) {
            int piv = c;
            for (int r = c + 1; r < n; ++r)
                if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
            for (int j = 0; j < 2 * n; ++j) std::swap(a[c][j], a[piv][j]);
            const double d = a[c][c];
            for (int j = 0; j < 2 * n; ++j) a[c][j] /= d;
            for (int r = 0; r < n; ++r)
                if (r != c) {
                    const double f = a[r][c];
                    for (int j = 0; j < 2 * n; ++j) a[r][j] -= f * a[c][j];
                }
        }
        for (int q = 0; q < n; ++q)
            for (int k = 0; k < n; ++k) {
                double v = 0.0;
                for (int d = 0; d < n; ++d) v += G[p - 1][q][d] * a[d][n + k];
                DQ[p - 1][q][k] = (float)v;
                DQd[p - 1][q][k] = v;
            }
    }
    CK(cudaMemcpyToSymbol(c_DQ32, DQ, sizeof DQ));
    CK(cudaMemcpyToSymbol(c_DQ64, DQd, sizeof DQd));
    g_tables_ready[dev] = true;
    return FG_OK;
}

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static int ensure_encode() {
    std::lock_guard<std::mutex> lk(g_init_mu);
    if (g_encode) return FG_OK;
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !fn)
        return fail(FG_CUDA_ERROR, "cuTensorMapEncodeTiled entry point not found");
    g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    return FG_OK;
}

// ---------------------------------------------------------------------------
// kernel configurations per order
// ---------------------------------------------------------------------------
template <int P> struct KCfg;
template <> struct KCfg<1> { static constexpr int WY = 4, S = 4, MINB = 3; };
template <> struct KCfg<2> { static constexpr int WY = 4, S = 3, MINB = 2; };
#ifndef FG_Q3_WY  // Q3 FP64 tile knobs (compile-time): row warps, qdata ring depth, CTAs/SM hint
#define FG_Q3_WY 2
#endif
#ifndef FG_Q3_S
#define FG_Q3_S 1
#endif
#ifndef FG_Q3_MINB
#define FG_Q3_MINB 1
#endif
template <> struct KCfg<3> { static constexpr int WY = FG_Q3_WY, S = FG_Q3_S, MINB = FG_Q3_MINB; };

static int cfg_wy(int p) { return p == 1 ? KCfg<1>::WY : p == 2 ? KCfg<2>::WY : KCfg<3>::WY; }

// ---------------------------------------------------------------------------
// the operator handle
// ---------------------------------------------------------------------------
struct fg_op {
    std::mutex mu;
    int device = 0;
    Grid g{};
    int ess_tags = 0, kind = 0, p = 0;
    int64_t N = 0, Nn = 0;
    double *qd = nullptr, *face = nullptr;
    double *xs = nullptr, *ys = nullptr;
    double *dinv = nullptr, *ones = nullptr;
    double *stage = nullptr;  // N values: contiguous device copy of a host vector
    // fused fix-up (FG_FUSED_FIXUP=1; off by default, fixup_kernel runs after each apply):
    // per-item arrival counters (FP64 applies, then FP32 applies), sized for the finest item
    // tiling (one layer per item)
    unsigned *fixcnt = nullptr;
    int64_t fixcnt_items = 0;
    bool fused_fixup = false;
    bool have_dinv = false;
    double lmax_est = 0.0;
    bool have_lmax = false;
    double *r = nullptr, *z = nullptr, *pv = nullptr, *ap = nullptr, *xw = nullptr, *bw = nullptr;
    double *cres = nullptr, *cd = nullptr, *ct = nullptr;
    double *cdk[CHEB_MAXD] = {};   // Chebyshev d_1 .. d_{s-1} (d_0 is cd)
    float *cdk32[CHEB_MAXD] = {};
    double *partials = nullptr;
    SolverState *st = nullptr;
    // FP32 operator data and inner-solve work vectors (iterative refinement)
    float *qd32 = nullptr, *face32 = nullptr, *dinv32 = nullptr;
    float *r32 = nullptr, *z32 = nullptr, *p32 = nullptr, *ap32 = nullptr, *e32 = nullptr,
          *b32 = nullptr, *cres32 = nullptr, *cd32 = nullptr, *ct32 = nullptr, *xs32 = nullptr,
          *ys32 = nullptr;
    int64_t qsize = 0;
    SolverState *st32 = nullptr;
    // affine-compressed quadrature data (fg_op_set_qdata_format), FP64 and FP32
    double *sd_u = nullptr, *sd_k1 = nullptr, *sd_w = nullptr;  // SDIRK-2 stepping
    // learned coarse correction (Q1 operators): coarse log kappa, network, scratch
    float *nn_lk = nullptr, *nn_rc = nullptr, *nn_oc = nullptr;
    std::vector<float *> nn_tmp;  // intermediate levels 1 .. nn_levels-1
    double *nn_scale = nullptr;
    int nn_levels = 1;  // coarsenings between the DOF lattice and the network volume
    cudaStream_t nn_stream = nullptr;          // high-priority side stream of the network
    cudaEvent_t nn_ev_r = nullptr, nn_ev_n = nullptr;
    bool nn_overlap = true;                    // network beside the smoother (FG_NN_OVERLAP=0: in line)
    fg_unet *nn = nullptr;
    // per-iteration device times (ms) of the plain and the learned
    // preconditioned iteration, per (precision, qdata format, Chebyshev degree)
    struct NnTimes { int ir, fmt, degree; double plain_ms, learned_ms; };
    std::vector<NnTimes> nn_times;
    int fmt = 0;
    // unstructured Hex8 mesh (fg_op_create_hex): element maps in the chunk
    // order, the chunk scatter's lists, essential-DOF mask; vectors are plain
    // (no pads)
    bool unstr = false;
    int64_t u_E = 0, u_chunks = 0, u_nshared = 0;
    int u_max_nu = 0;
    int32_t *u_dofs = nullptr;
    uint8_t *u_ess = nullptr;
    uint64_t *u_emsk = nullptr;  // [E] essential local DOFs of each element (bit k)
    int32_t *u_cu_off = nullptr, *u_cu_dof = nullptr, *u_cu_pid = nullptr, *u_cu_soff = nullptr;
    int32_t *u_sh_dof = nullptr, *u_sh_off = nullptr;
    uint16_t *u_cu_slots = nullptr;
    double *u_part = nullptr;  // partials of the shared DOFs (FP64 or FP32 applies)
    double *qa64 = nullptr;
    float *qa32 = nullptr;
    int *d_err = nullptr;
    unsigned *bar = nullptr;  // grid-barrier counters of the fused PCG iteration kernel
    bool fused_pcg = true;    // one cooperative launch per Jacobi-PCG iteration (FG_FUSED_PCG=0: three)
    bool pipelined = true;    // host-memory applies pipelined over z ranges (FG_PIPELINED_APPLY=0: not)
    uint64_t wait_ns = 0;  // limit of the apply kernels' device-side waits (0: 1 s)
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t cap_stream = nullptr;  // private stream for CUDA-graph capture
    // pipelined host-memory applies: upload and download streams, per-range events
    cudaStream_t s_in = nullptr, s_out = nullptr;
    std::vector<cudaEvent_t> ev_in, ev_out;
    bool graphs = true;                 // replay solver chunks as CUDA graphs
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

static void free_op(fg_op *op) {
    if (!op) return;
    cudaSetDevice(op->device);
    if (op->stream) cudaStreamSynchronize(op->stream);
    double *bufs[] = {op->qd, op->face, op->xs, op->ys, op->dinv, op->ones, op->r, op->z, op->pv, op->ap,
                      op->xw, op->bw, op->cres, op->cd, op->ct, op->partials, op->stage};
    if (op->fixcnt) cudaFree(op->fixcnt);
    if (op->u_dofs) cudaFree(op->u_dofs);
    if (op->u_ess) cudaFree(op->u_ess);
    {
        void *u[] = {op->u_emsk, op->u_cu_off, op->u_cu_dof, op->u_cu_pid, op->u_cu_soff, op->u_sh_dof, op->u_sh_off,
                     op->u_cu_slots, op->u_part};
        for (void *q : u)
            if (q) cudaFree(q);
    }
    for (int k = 0; k < CHEB_MAXD; ++k) {
        if (op->cdk[k]) cudaFree(op->cdk[k]);
        if (op->cdk32[k]) cudaFree(op->cdk32[k]);
    }
    for (double *b : bufs)
        if (b) cudaFree(b);
    float *fb[] = {op->qd32, op->face32, op->dinv32, op->r32, op->z32, op->p32, op->ap32, op->e32,
                   op->b32, op->cres32, op->cd32, op->ct32, op->xs32, op->ys32};
    for (float *b : fb)
        if (b) cudaFree(b);
    if (op->st32) cudaFree(op->st32);
    if (op->qa64) cudaFree(op->qa64);
    if (op->sd_u) cudaFree(op->sd_u);
    if (op->nn_lk) cudaFree(op->nn_lk);
    if (op->nn_rc) cudaFree(op->nn_rc);
    if (op->nn_oc) cudaFree(op->nn_oc);
    for (float *t : op->nn_tmp) cudaFree(t);
    if (op->nn_scale) cudaFree(op->nn_scale);
    if (op->sd_k1) cudaFree(op->sd_k1);
    if (op->sd_w) cudaFree(op->sd_w);
    if (op->qa32) cudaFree(op->qa32);
    if (op->st) cudaFree(op->st);
    if (op->bar) cudaFree(op->bar);
    if (op->d_err) cudaFree(op->d_err);
    if (op->ev0) cudaEventDestroy(op->ev0);
    if (op->ev1) cudaEventDestroy(op->ev1);
    if (op->own_stream && op->stream) cudaStreamDestroy(op->stream);
    if (op->cap_stream) cudaStreamDestroy(op->cap_stream);
    if (op->s_in) cudaStreamDestroy(op->s_in);
    if (op->s_out) cudaStreamDestroy(op->s_out);
    for (cudaEvent_t e : op->ev_in) cudaEventDestroy(e);
    for (cudaEvent_t e : op->ev_out) cudaEventDestroy(e);
    if (op->nn_stream) cudaStreamDestroy(op->nn_stream);
    if (op->nn_ev_r) cudaEventDestroy(op->nn_ev_r);
    if (op->nn_ev_n) cudaEventDestroy(op->nn_ev_n);
    delete op;
}

template <typename T> static int alloc_vec(T **p, int64_t n) {
    CK(cudaMalloc(p, sizeof(T) * std::max<int64_t>(n, 1)));
    CK(cudaMemset(*p, 0, sizeof(T) * std::max<int64_t>(n, 1)));
    FG_LEGACY_FENCE();
    return FG_OK;
}

#include "hex_host.cuh"

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <int P> struct KCfg32;  // FP32 apply: same tile (WY) as FP64, deeper rings
template <> struct KCfg32<1> { static constexpr int WY = 4, S = 6, MINB = 4; };
#ifndef FG_F32_Q2_S  // FP32 Q2 full-format qdata ring depth (stages of one quadrature column per warp)
#define FG_F32_Q2_S 4
#endif
#ifndef FG_F32_Q2_MINB  // FP32 Q2 CTAs/SM hint
#define FG_F32_Q2_MINB 3
#endif
template <> struct KCfg32<2> { static constexpr int WY = 4, S = FG_F32_Q2_S, MINB = FG_F32_Q2_MINB; };
#ifndef FG_F32_Q3_S  // FP32 Q3 qdata ring depth and CTAs/SM hint
#define FG_F32_Q3_S 3
#endif
#ifndef FG_F32_Q3_MINB
#define FG_F32_Q3_MINB 2
#endif
template <> struct KCfg32<3> { static constexpr int WY = FG_Q3_WY, S = FG_F32_Q3_S, MINB = FG_F32_Q3_MINB; };
#ifndef FG_F32_Q2_AS  // FP32 Q2 affine-format qdata ring depth (stages of one element layer per warp)
#define FG_F32_Q2_AS 1
#endif
#ifndef FG_F32_Q2_AMINB  // FP32 Q2 affine-format CTAs/SM hint (the 1-deep ring leaves room for 5)
#define FG_F32_Q2_AMINB 5
#endif
// ring depth of the affine format: one element layer per stage
#ifndef FG_F32_Q3_AS  // FP32 Q3 affine-format qdata ring depth (1: 4 CTAs per SM instead of 3)
#define FG_F32_Q3_AS 1
#endif
#ifndef FG_AFFINE_AS  // affine-format qdata ring depth of the other orders and precisions
#define FG_AFFINE_AS 2
#endif
template <int P, typename T> constexpr int affine_stages() {
    return std::is_same<T, float>::value ? (P == 2 ? FG_F32_Q2_AS : (P == 3 ? FG_F32_Q3_AS : FG_AFFINE_AS))
                                         : FG_AFFINE_AS;
}
// CTAs/SM hint of an apply kernel
template <int P, typename T, int FMT, int MINB> constexpr int apply_minb() {
    return (FMT == 1 && P == 2 && std::is_same<T, float>::value) ? FG_F32_Q2_AMINB : MINB;
}
template <int P, typename T> struct KC;
template <int P> struct KC<P, double> : KCfg<P> {};
template <int P> struct KC<P, float> : KCfg32<P> {};

template <typename T> struct TmapType;
template <> struct TmapType<double> { static constexpr CUtensorMapDataType v = CU_TENSOR_MAP_DATA_TYPE_FLOAT64; };
template <> struct TmapType<float> { static constexpr CUtensorMapDataType v = CU_TENSOR_MAP_DATA_TYPE_FLOAT32; };

template <int P, int OPK, typename T, int FMT>
static int launch_apply_t(fg_op *op, const Grid &g, const T *qd, T *face, const T *x, T *y,
                          int accumulate, const int *skip, unsigned *fixcnt = nullptr, int item0 = 0,
                          int nitems = -1) {
    using C = KC<P, T>;
    static_assert(C::WY == KCfg<P>::WY, "FP32 and FP64 share the item tiling");
    constexpr int S = FMT == 0 ? C::S : affine_stages<P, T>();  // affine format: one element layer per stage
    using SM = ApplySmem<P, T, C::WY, S, stage_elems<P, OPK, FMT>() / 32>;
    // per device, set once; handles on several host threads may race here, and
    // setting the same attribute twice is harmless
    static std::atomic<bool> attr_set[64];
    auto kern = pa_apply_kernel<P, OPK, T, C::WY, S, apply_minb<P, T, FMT, C::MINB>(), FMT>;
    if (!attr_set[op->device].load(std::memory_order_acquire)) {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SM::bytes));
        attr_set[op->device].store(true, std::memory_order_release);
    }
    CUtensorMap tmap;
    cuuint64_t gdim[3] = {(cuuint64_t)g.NI, (cuuint64_t)g.NJ, (cuuint64_t)g.NK};
    cuuint64_t gstr[2] = {(cuuint64_t)g.NIp * sizeof(T), (cuuint64_t)g.NIp * g.NJ * sizeof(T)};
    cuuint32_t box[3] = {(cuuint32_t)SM::XW, (cuuint32_t)SM::RY, (cuuint32_t)(P + 1)};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult cr = g_encode(&tmap, TmapType<T>::v, 3, const_cast<T *>(x), gdim, gstr, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return fail(FG_CUDA_ERROR, "cuTensorMapEncodeTiled failed (%d)", (int)cr);
    ApplyArgs<T> A{g, qd, y, face, accumulate, op->d_err, skip, fixcnt, op->wait_ns, item0};
    kern<<<nitems < 0 ? g.n_items() : nitems, C::WY * 32, SM::bytes, op->stream>>>(tmap, A);
    CK(cudaGetLastError());
    return FG_OK;
}

template <typename T> static const T *qdata_of(fg_op *op);
template <> const double *qdata_of<double>(fg_op *op) { return op->fmt ? op->qa64 : op->qd; }
template <> const float *qdata_of<float>(fg_op *op) { return op->fmt ? op->qa32 : op->qd32; }

template <int P, typename T>
static int launch_apply_p(fg_op *op, const Grid &g, const T *, T *face, const T *x, T *y,
                          int accumulate, const int *skip, unsigned *fixcnt, int item0 = 0, int nitems = -1) {
    const T *qd = qdata_of<T>(op);
    if (!qd) return fail(FG_INVALID_ARGUMENT, "quadrature data for this precision/format not built");
    if (op->fmt == 0) {
        switch (op->kind) {
        case FG_MASS: return launch_apply_t<P, 1, T, 0>(op, g, qd, face, x, y, accumulate, skip, fixcnt, item0, nitems);
        case FG_DIFF: return launch_apply_t<P, 2, T, 0>(op, g, qd, face, x, y, accumulate, skip, fixcnt, item0, nitems);
        default: return launch_apply_t<P, 3, T, 0>(op, g, qd, face, x, y, accumulate, skip, fixcnt, item0, nitems);
        }
    }
    switch (op->kind) {
    case FG_MASS: return launch_apply_t<P, 1, T, 1>(op, g, qd, face, x, y, accumulate, skip, fixcnt, item0, nitems);
    case FG_DIFF: return launch_apply_t<P, 2, T, 1>(op, g, qd, face, x, y, accumulate, skip, fixcnt, item0, nitems);
    default: return launch_apply_t<P, 3, T, 1>(op, g, qd, face, x, y, accumulate, skip, fixcnt, item0, nitems);
    }
}

static dim3 fixup_grid(const Grid &g) { return dim3(fixup_rows(g)); }

template <typename T>
static int launch_fixup(fg_op *op, const Grid &g, T *y, const T *face, const int *skip) {
    const dim3 grid = fixup_grid(g);
    if (grid.x == 0) return FG_OK;
    fixup_kernel<T><<<grid, 128, 0, op->stream>>>(g, y, face, skip);
    CK(cudaGetLastError());
    return FG_OK;
}

// Arrival counters of the fused fix-up for an apply into the handle's own face
// buffer of this precision (one set per precision, so an FP64 and an FP32
// apply never share them), or null: the separate fixup_kernel.
template <typename T> static unsigned *fixcnt_for(fg_op *op, const T *face) {
    if (!op->fused_fixup || !op->fixcnt) return nullptr;
    if (std::is_same<T, double>::value && (const void *)face == (const void *)op->face) return op->fixcnt;
    if (std::is_same<T, float>::value && (const void *)face == (const void *)op->face32)
        return op->fixcnt + op->fixcnt_items;
    return nullptr;
}

// y (+)= A x on native vectors with the given precision's quadrature data.
template <typename T>
static int apply_native_t(fg_op *op, const T *qd, T *face, const T *x, T *y, int accumulate,
                          int constrained, const int *skip) {
    if (op->unstr) return hex_apply<T>(op, qd, x, y, accumulate, constrained, skip);
    unsigned *fixcnt = fixcnt_for<T>(op, face);
    Grid g = op->g;
    g.ess = constrained ? op->ess_tags : 0;
    int rc;
    switch (op->p) {
    case 1: rc = launch_apply_p<1, T>(op, g, qd, face, x, y, accumulate, skip, fixcnt); break;
    case 2: rc = launch_apply_p<2, T>(op, g, qd, face, x, y, accumulate, skip, fixcnt); break;
    default: rc = launch_apply_p<3, T>(op, g, qd, face, x, y, accumulate, skip, fixcnt); break;
    }
    if (rc || fixcnt) return rc;
    return launch_fixup<T>(op, g, y, face, skip);
}

static int apply_native(fg_op *op, const double *x, double *y, int accumulate, int constrained,
                        const int *skip) {
    return apply_native_t<double>(op, op->qd, op->face, x, y, accumulate, constrained, skip);
}

template <int P, int OPK> static int launch_diag_t(fg_op *op, const Grid &g, double *y) {
    constexpr int WY = KCfg<P>::WY;
    ApplyArgs<double> A{g, op->qd, y, op->face, 0, op->d_err, nullptr};
    pa_diag_kernel<P, OPK, double, WY><<<g.n_items(), WY * 32, 0, op->stream>>>(A);
    CK(cudaGetLastError());
    return FG_OK;
}
template <int P> static int launch_diag_p(fg_op *op, const Grid &g, double *y) {
    switch (op->kind) {
    case FG_MASS: return launch_diag_t<P, 1>(op, g, y);
    case FG_DIFF: return launch_diag_t<P, 2>(op, g, y);
    default: return launch_diag_t<P, 3>(op, g, y);
    }
}
static int diag_native(fg_op *op, double *y, int constrained) {
    if (op->unstr) return hex_diag(op, y, constrained);
    Grid g = op->g;
    g.ess = constrained ? op->ess_tags : 0;
    int rc;
    switch (op->p) {
    case 1: rc = launch_diag_p<1>(op, g, y); break;
    case 2: rc = launch_diag_p<2>(op, g, y); break;
    default: rc = launch_diag_p<3>(op, g, y); break;
    }
    if (rc) return rc;
    return launch_fixup<double>(op, g, y, op->face, nullptr);
}

template <int P, int OPK, typename T = double>
static int launch_setup_t(fg_op *op, SetupArgs &S, T *qd = nullptr) {
    const int64_t total = (int64_t)op->g.nx * op->g.ny * op->g.nz * (P + 1) * (P + 1) * (P + 1);
    const int threads = 256;
    const int blocks = (int)std::min<int64_t>((total + threads - 1) / threads, 148 * 32);
    qdata_setup_kernel<P, OPK, T><<<blocks, threads, 0, op->stream>>>(S, qd ? qd : (T *)op->qd);
    CK(cudaGetLastError());
    return FG_OK;
}
template <int P> static int launch_setup_p(fg_op *op, SetupArgs &S, int64_t *qsize) {
    switch (op->kind) {
    case FG_MASS: *qsize = qd_size<P, 1>(op->g); break;
    case FG_DIFF: *qsize = qd_size<P, 2>(op->g); break;
    default: *qsize = qd_size<P, 3>(op->g); break;
    }
    if (!op->qd) {
        int rc = alloc_vec(&op->qd, *qsize);
        if (rc) return rc;
        return FG_OK;
    }
    switch (op->kind) {
    case FG_MASS: return launch_setup_t<P, 1>(op, S);
    case FG_DIFF: return launch_setup_t<P, 2>(op, S);
    default: return launch_setup_t<P, 3>(op, S);
    }
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

FG_API void fg_cfg_default(fg_cfg *c) {
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->rtol = 1e-8;
    c->atol = 0.0;
    c->max_iter = 1000;
    c->print_level = 0;
    c->precond = FG_PC_JACOBI;
    c->cheb_degree = 4;
    c->precision = FG_FP64;
    c->power_iters = 20;
    c->lmax = 0.0;
    c->lmin_ratio = 30.0;
    c->lmax_safety = 1.1;
    c->inner_rtol = 0.1;
    c->check_interval = 10;
}

FG_API int fg_last_error(char *buf, size_t n) {
    if (buf && n) {
        std::strncpy(buf, t_last_msg.c_str(), n - 1);
        buf[n - 1] = 0;
    }
    return t_last_status;
}

FG_API int fg_op_create(const fg_mesh *mesh, int order, int nq1d, int kind, double c_mass,
                        double c_diff, const double *kappa_q, double kappa_const,
                        const double *rho_q, double rho_const, int ess_tags, fg_op **out) {
    t_last_status = FG_OK;
    if (!out) return fail(FG_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!mesh || mesh->nx < 1 || mesh->ny < 1 || mesh->nz < 1)
        return fail(FG_INVALID_ARGUMENT, "mesh must have at least one element per direction");
    if (order < 1 || order > FG_MAXP)
        return fail(FG_UNSUPPORTED, "unsupported order %d (supported: 1..%d)", order, FG_MAXP);
    if (nq1d != order + 1)
        return fail(FG_UNSUPPORTED, "nq1d must be order+1 (hex_rule(2p+1)), got %d", nq1d);
    if (kind < 1 || kind > 3) return fail(FG_INVALID_ARGUMENT, "bad operator kind %d", kind);
    if (ess_tags < 0 || ess_tags > 63) return fail(FG_INVALID_ARGUMENT, "bad ess_tags %d", ess_tags);
    const int64_t NI = (int64_t)mesh->nx * order + 1, NJ = (int64_t)mesh->ny * order + 1,
                  NK = (int64_t)mesh->nz * order + 1;
    if (NI * NJ * NK > ((int64_t)1 << 40) || NI > (1 << 20) || NJ > (1 << 20) || NK > (1 << 20))
        return fail(FG_INVALID_ARGUMENT, "mesh too large");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    int rc = ensure_tables(dev);
    if (rc) return rc;
    if ((rc = ensure_encode())) return rc;

    fg_op *op = new fg_op();
    op->device = dev;
    op->kind = kind;
    op->p = order;
    op->ess_tags = ess_tags;
    Grid &g = op->g;
    g.nx = mesh->nx; g.ny = mesh->ny; g.nz = mesh->nz; g.p = order;
    g.NI = (int)NI; g.NJ = (int)NJ; g.NK = (int)NK;
    g.NIp = round_up((int)NI, 4);
    g.WY = cfg_wy(order);
    g.ntx = (g.nx + 31) / 32;
    g.nty = (g.ny + g.WY - 1) / g.WY;
    // layers per item: as many as keep >= 4 items per SM slot on a 148-SM part
    int TZ = 8;
    while (TZ > 1 && (int64_t)g.ntx * g.nty * ((g.nz + TZ - 1) / TZ) < 148 * 4) TZ /= 2;
    g.TZ = TZ;
    g.ntz = (g.nz + TZ - 1) / TZ;
    g.ess = 0;
    op->N = NI * NJ * NK;
    op->Nn = (int64_t)g.NIp * NJ * NK;

    auto bail = [&](int s) { free_op(op); return s; };
    if (cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(FG_CUDA_ERROR, "cudaStreamCreate failed"));
    op->own_stream = true;
    {
        const char *e = std::getenv("FG_SOLVER_GRAPHS");
        op->graphs = !(e && e[0] == '0');
        const char *o = std::getenv("FG_NN_OVERLAP");
        op->nn_overlap = !(o && o[0] == '0');
        const char *f = std::getenv("FG_FUSED_FIXUP");
        op->fused_fixup = f && f[0] == '1';
        const char *fp = std::getenv("FG_FUSED_PCG");
        op->fused_pcg = !(fp && fp[0] == '0');
        const char *pp = std::getenv("FG_PIPELINED_APPLY");
        op->pipelined = !(pp && pp[0] == '0');
    }
    if (cudaMalloc(&op->d_err, sizeof(int)) != cudaSuccess || cudaMemset(op->d_err, 0, sizeof(int)))
        return bail(fail(FG_CUDA_ERROR, "cudaMalloc failed"));
    if (cudaMalloc(&op->st, sizeof(SolverState)) != cudaSuccess ||
        cudaMemset(op->st, 0, sizeof(SolverState)) != cudaSuccess)
        return bail(fail(FG_CUDA_ERROR, "cudaMalloc failed"));
    if ((rc = alloc_vec(&op->face, (int64_t)g.n_items() * g.face_stride()))) return bail(rc);
    op->fixcnt_items = (int64_t)g.ntx * g.nty * g.nz;  // items at one layer each: any tiling fits
    if ((rc = alloc_vec(&op->fixcnt, 2 * op->fixcnt_items))) return bail(rc);
    if ((rc = alloc_vec(&op->xs, op->Nn)) || (rc = alloc_vec(&op->ys, op->Nn))) return bail(rc);
    if ((rc = alloc_vec(&op->partials, VEC_GRID * 4))) return bail(rc);
    cudaEventCreate(&op->ev0);
    cudaEventCreate(&op->ev1);

    // inputs for the quadrature-data build
    const int64_t E = (int64_t)g.nx * g.ny * g.nz;
    const int Q3 = (order + 1) * (order + 1) * (order + 1);
    double *d_vc = nullptr, *d_kq = nullptr, *d_rq = nullptr;
    auto cleanup_in = [&]() {
        if (d_vc) cudaFree(d_vc);
        if (d_kq) cudaFree(d_kq);
        if (d_rq) cudaFree(d_rq);
    };
    if (mesh->vcoord) {
        const size_t nb = sizeof(double) * 3 * (size_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
        if (cudaMalloc(&d_vc, nb) || cudaMemcpy(d_vc, mesh->vcoord, nb, cudaMemcpyDefault)) {
            cleanup_in();
            return bail(fail(FG_CUDA_ERROR, "vertex upload failed"));
        }
    }
    if (kappa_q) {
        const size_t nb = sizeof(double) * E * Q3;
        if (cudaMalloc(&d_kq, nb) || cudaMemcpy(d_kq, kappa_q, nb, cudaMemcpyDefault)) {
            cleanup_in();
            return bail(fail(FG_CUDA_ERROR, "kappa upload failed"));
        }
    }
    if (rho_q) {
        const size_t nb = sizeof(double) * E * Q3;
        if (cudaMalloc(&d_rq, nb) || cudaMemcpy(d_rq, rho_q, nb, cudaMemcpyDefault)) {
            cleanup_in();
            return bail(fail(FG_CUDA_ERROR, "rho upload failed"));
        }
    }
    if (cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess) {  // d_err/st memsets, uploads
        cleanup_in();
        return bail(fail(FG_CUDA_ERROR, "set-up copies failed"));
    }
    SetupArgs S{};
    S.g = g;
    S.vcoord = d_vc;
    S.kappa_q = d_kq;
    S.rho_q = d_rq;
    S.kappa_c = kappa_const;
    S.rho_c = rho_const;
    S.c_m = c_mass;
    S.c_k = c_diff;
    gauss_legendre(order + 1, S.gx, S.gw);
    S.err = op->d_err;
    int64_t qsize = 0;
    for (int pass = 0; pass < 2 && !rc; ++pass) {  // pass 0 allocates, pass 1 launches
        switch (order) {
        case 1: rc = launch_setup_p<1>(op, S, &qsize); break;
        case 2: rc = launch_setup_p<2>(op, S, &qsize); break;
        default: rc = launch_setup_p<3>(op, S, &qsize); break;
        }
    }
    op->qsize = qsize;
    if (!rc && cudaStreamSynchronize(op->stream) != cudaSuccess)
        rc = fail(FG_CUDA_ERROR, "qdata setup failed: %s", cudaGetErrorString(cudaGetLastError()));
    cleanup_in();
    if (rc) return bail(rc);
    int herr = 0;
    cudaMemcpy(&herr, op->d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (herr & FG_DERR_BOUNDS) return bail(fail(FG_BOUNDS, "degenerate element (det J = 0)"));
    *out = op;
    return FG_OK;
}

FG_API void fg_op_destroy(fg_op *op) { free_op(op); }

FG_API int64_t fg_op_ndofs(const fg_op *op) { return op ? op->N : -1; }

FG_API int64_t fg_op_native_len(const fg_op *op) { return op ? op->Nn : -1; }

FG_API int fg_op_layout(const fg_op *op, int64_t dims[4]) {
    if (!op || !dims) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    dims[0] = op->g.NI; dims[1] = op->g.NJ; dims[2] = op->g.NK; dims[3] = op->g.NIp;
    return FG_OK;
}

FG_API int fg_op_set_stream(fg_op *op, void *stream) {
    if (!op) return fail(FG_INVALID_ARGUMENT, "NULL op");
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    CK(cudaStreamSynchronize(op->stream));
    if (op->own_stream) cudaStreamDestroy(op->stream);
    op->own_stream = false;
    op->stream = reinterpret_cast<cudaStream_t>(stream);
    return FG_OK;
}

FG_API int fg_op_set_wait_limit(fg_op *op, double seconds) {
    if (!op) return fail(FG_INVALID_ARGUMENT, "NULL operator");
    if (!(seconds == seconds)) return fail(FG_INVALID_ARGUMENT, "wait limit is NaN");
    std::lock_guard<std::mutex> lk(op->mu);
    op->wait_ns = seconds <= 0.0 ? 0 : std::max<uint64_t>(1, (uint64_t)std::min(seconds * 1e9, 6e10));
    t_last_status = FG_OK;
    return FG_OK;
}

static int check_device_error(fg_op *op) {
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, op->d_err, sizeof(int), cudaMemcpyDeviceToHost, op->stream));
    CK(cudaStreamSynchronize(op->stream));
    if (herr) {
        cudaMemsetAsync(op->d_err, 0, sizeof(int), op->stream);
        if (op->bar) cudaMemsetAsync(op->bar, 0, 2 * sizeof(unsigned), op->stream);  // after a barrier timeout
        if (herr & FG_DERR_TIMEOUT) return fail(FG_DEVICE_TIMEOUT, "device-side wait timed out");
        return fail(FG_BOUNDS, "device-side bounds error");
    }
    return FG_OK;
}

FG_API int fg_op_check(fg_op *op) {
    if (!op) return fail(FG_INVALID_ARGUMENT, "NULL op");
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    return check_device_error(op);
}

}  // extern "C"

// Host vectors cross PCIe as one contiguous copy through the handle's staging
// buffer; the change of row pitch (NI <-> NIp) is a device-to-device 2-D copy.
// A 2-D copy straight from or to host memory moves one DOF row per transfer and
// ran at about half the contiguous PCIe rate.
template <typename T> static int stage_of(fg_op *op, T **st) {
    static_assert(sizeof(T) <= sizeof(double), "staging holds N doubles");
    if (!op->stage) {
        int rc = alloc_vec(&op->stage, op->N);
        if (rc) return rc;
    }
    *st = reinterpret_cast<T *>(op->stage);
    return FG_OK;
}
// rows x w values between pitches sp and dp (elements) on `s`, by k_repitch
template <typename T>
static int repitch(const T *src, int64_t sp, T *dst, int64_t dp, int w, int64_t rows, cudaStream_t s) {
    if (rows <= 0) return FG_OK;
    const int64_t blocks = std::min<int64_t>((rows + 7) / 8, 148 * 16);
    k_repitch<T><<<(unsigned)blocks, 256, 0, s>>>(src, sp, dst, dp, w, rows);
    CK(cudaGetLastError());
    return FG_OK;
}

template <typename T> static int to_native_t(fg_op *op, T *dst, const T *src, int mem) {
    const Grid &g = op->g;
    if (mem == FG_HOST) {
        T *st = nullptr;
        int rc = stage_of(op, &st);
        if (rc) return rc;
        CK(cudaMemcpyAsync(st, src, sizeof(T) * op->N, cudaMemcpyHostToDevice, op->stream));
        src = st;
    }
    return repitch<T>(src, g.NI, dst, g.NIp, g.NI, (int64_t)g.NJ * g.NK, op->stream);
}
template <typename T> static int from_native_t(fg_op *op, T *dst, const T *src, int mem) {
    const Grid &g = op->g;
    T *out = dst;
    if (mem == FG_HOST) {
        int rc = stage_of(op, &out);
        if (rc) return rc;
    }
    int rc;
    if ((rc = repitch<T>(src, g.NIp, out, g.NI, g.NI, (int64_t)g.NJ * g.NK, op->stream))) return rc;
    if (mem == FG_HOST)
        CK(cudaMemcpyAsync(dst, out, sizeof(T) * op->N, cudaMemcpyDeviceToHost, op->stream));
    return FG_OK;
}
static int to_native(fg_op *op, double *dst, const double *src, int mem) {
    return to_native_t<double>(op, dst, src, mem);
}
static int from_native(fg_op *op, double *dst, const double *src, int mem) {
    return from_native_t<double>(op, dst, src, mem);
}

// y = A x for host vectors on a box, pipelined over ranges of item layers in
// z: the upload of range r+1's DOF planes, the apply and fix-up of range r and
// the download of range r-1's finished planes run at the same time (PCIe moves
// data both ways at once).  Range r's items need the planes [A_r, A_{r+1}]
// (A_r = first plane of its item layers); its fix-up completes the planes
// [A_r, A_{r+1}), whose owners are its items (plane A_{r+1} belongs to the next
// range, which adds this range's face partials in its own fix-up).  Upload
// chunk r holds the planes (A_r, A_{r+1}] (chunk 0 from plane 0), so range r
// can start once chunks 0..r have arrived.  The staging buffer holds x planes
// on the way in and y planes on the way out: a y range is packed only after
// the x planes it overlaps were repacked, and uploads never touch it again.
static int apply_host_pipelined(fg_op *op, const double *x, double *y, int constrained) {
    Grid g = op->g;
    g.ess = constrained ? op->ess_tags : 0;
    static const int max_ranges = [] {  // FG_PIPE_RANGES: z ranges of the pipeline (default 16)
        const char *e = std::getenv("FG_PIPE_RANGES");
        const int v = e ? std::atoi(e) : 16;
        return v >= 1 && v <= 256 ? v : 16;
    }();
    const int R = std::min(g.ntz, max_ranges);
    double *st = nullptr;
    int rc = stage_of(op, &st);
    if (rc) return rc;
    if (!op->s_in) {
        CK(cudaStreamCreateWithFlags(&op->s_in, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&op->s_out, cudaStreamNonBlocking));
    }
    while ((int)op->ev_in.size() < R) {
        cudaEvent_t a, b;
        CK(cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
        op->ev_in.push_back(a);
        op->ev_out.push_back(b);
    }
    const int SZe = g.TZ * g.p;
    const int64_t plane = (int64_t)g.NI * g.NJ;  // plain values per DOF plane
    std::vector<int> t0(R + 1), A(R + 1);
    for (int r = 0; r <= R; ++r) t0[r] = (int)((int64_t)g.ntz * r / R);
    for (int r = 0; r < R; ++r) A[r] = t0[r] * SZe;
    A[R] = g.NK - 1;
    // the caller's stream has to see the handle's earlier work first
    CK(cudaEventRecord(op->ev_out[0], op->stream));
    CK(cudaStreamWaitEvent(op->s_in, op->ev_out[0], 0));
    for (int r = 0; r < R; ++r) {  // uploads, in order on the upload stream
        const int lo = r == 0 ? 0 : A[r] + 1, hi = A[r + 1] + 1;
        CK(cudaMemcpyAsync(st + lo * plane, x + lo * plane, sizeof(double) * plane * (hi - lo),
                           cudaMemcpyHostToDevice, op->s_in));
        CK(cudaEventRecord(op->ev_in[r], op->s_in));
    }
    const int items_per_layer = g.ntx * g.nty;
    for (int r = 0; r < R; ++r) {
        const int lo = r == 0 ? 0 : A[r] + 1, hi = A[r + 1] + 1;
        CK(cudaStreamWaitEvent(op->stream, op->ev_in[r], 0));
        if ((rc = repitch<double>(st + lo * plane, g.NI, op->xs + (int64_t)lo * g.NJ * g.NIp, g.NIp, g.NI,
                                  (int64_t)g.NJ * (hi - lo), op->stream)))
            return rc;
        const int i0 = t0[r] * items_per_layer, ni = (t0[r + 1] - t0[r]) * items_per_layer;
        switch (op->p) {
        case 1: rc = launch_apply_p<1, double>(op, g, op->qd, op->face, op->xs, op->ys, 0, nullptr, nullptr, i0, ni); break;
        case 2: rc = launch_apply_p<2, double>(op, g, op->qd, op->face, op->xs, op->ys, 0, nullptr, nullptr, i0, ni); break;
        default: rc = launch_apply_p<3, double>(op, g, op->qd, op->face, op->xs, op->ys, 0, nullptr, nullptr, i0, ni); break;
        }
        if (rc) return rc;
        // fix-up of the planes this range owns
        const int Ka = A[r], Kb = r == R - 1 ? g.NK : A[r + 1];
        int pl0 = 0, npl = 0;
        for (int pl = 0; pl < g.ntz - 1; ++pl) {
            const int K = (pl + 1) * SZe;
            if (K >= Ka && K < Kb) {
                if (!npl) pl0 = pl;
                ++npl;
            }
        }
        const int rows = (g.ntx - 1 + g.nty - 1) * (Kb - Ka) + npl * g.NJ;
        if (rows > 0) {
            fixup_range_kernel<double><<<rows, 128, 0, op->stream>>>(g, op->ys, op->face, Ka, Kb, pl0);
            CK(cudaGetLastError());
        }
        if ((rc = repitch<double>(op->ys + (int64_t)Ka * g.NJ * g.NIp, g.NIp, st + Ka * plane, g.NI, g.NI,
                                  (int64_t)g.NJ * (Kb - Ka), op->stream)))
            return rc;
        CK(cudaEventRecord(op->ev_out[r], op->stream));
        CK(cudaStreamWaitEvent(op->s_out, op->ev_out[r], 0));
        CK(cudaMemcpyAsync(y + Ka * plane, st + Ka * plane, sizeof(double) * plane * (Kb - Ka),
                           cudaMemcpyDeviceToHost, op->s_out));
    }
    // the handle's stream ends after the last download
    CK(cudaEventRecord(op->ev_in[0], op->s_out));
    CK(cudaStreamWaitEvent(op->stream, op->ev_in[0], 0));
    return FG_OK;
}

extern "C" {

FG_API int fg_op_apply(fg_op *op, const double *x, double *y, int accumulate, int constrained,
                       int mem) {
    if (!op || !x || !y) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (mem != FG_HOST && mem != FG_DEVICE) return fail(FG_INVALID_ARGUMENT, "bad mem %d", mem);
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    int rc;
    if (mem == FG_HOST && !accumulate && !op->unstr && !op->fused_fixup && op->g.ntz >= 2 && op->pipelined) {
        if ((rc = apply_host_pipelined(op, x, y, constrained))) return rc;
        return check_device_error(op);
    }
    if ((rc = to_native(op, op->xs, x, mem))) return rc;
    if (accumulate && (rc = to_native(op, op->ys, y, mem))) return rc;
    if ((rc = apply_native(op, op->xs, op->ys, accumulate, constrained, nullptr))) return rc;
    if ((rc = from_native(op, y, op->ys, mem))) return rc;
    return check_device_error(op);
}

FG_API int fg_op_apply_native(fg_op *op, const double *x, double *y, int accumulate,
                              int constrained) {
    if (!op || !x || !y) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (x == y) return fail(FG_INVALID_ARGUMENT, "x and y must not alias");
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    return apply_native(op, x, y, accumulate, constrained, nullptr);
}

FG_API int fg_op_diagonal(fg_op *op, double *d, int constrained, int mem) {
    if (!op || !d) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    int rc;
    if ((rc = diag_native(op, op->ys, constrained))) return rc;
    if ((rc = from_native(op, d, op->ys, mem))) return rc;
    return check_device_error(op);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// PCG
// ---------------------------------------------------------------------------
template <int P, int OPK, typename T> static void launch_compress(fg_op *op, T *dst) {
    const int64_t total = (int64_t)op->g.nx * op->g.ny * op->g.nz * (P + 1) * (P + 1) * (P + 1);
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
    qdata_compress_kernel<P, OPK, T><<<blocks, 256, 0, op->stream>>>(op->g, op->qd, dst, op->d_err);
}
template <int P, typename T> static void launch_compress_p(fg_op *op, T *dst) {
    switch (op->kind) {
    case FG_MASS: launch_compress<P, 1, T>(op, dst); break;
    case FG_DIFF: launch_compress<P, 2, T>(op, dst); break;
    default: launch_compress<P, 3, T>(op, dst); break;
    }
}
template <typename T> static int64_t affine_size(fg_op *op) {
    auto sz = [&](auto pk, auto ok) -> int64_t {
        constexpr int P = decltype(pk)::value, OPK = decltype(ok)::value;
        return qd_size_fmt<P, OPK, 1>(op->g);
    };
    using I1 = std::integral_constant<int, 1>;
    using I2 = std::integral_constant<int, 2>;
    using I3 = std::integral_constant<int, 3>;
    const int k = op->kind;
    switch (op->p) {
    case 1: return k == 1 ? sz(I1{}, I1{}) : k == 2 ? sz(I1{}, I2{}) : sz(I1{}, I3{});
    case 2: return k == 1 ? sz(I2{}, I1{}) : k == 2 ? sz(I2{}, I2{}) : sz(I2{}, I3{});
    default: return k == 1 ? sz(I3{}, I1{}) : k == 2 ? sz(I3{}, I2{}) : sz(I3{}, I3{});
    }
}
// Affine-compressed quadrature data in precision T, derived from the full FP64
// data; refused (FG_UNSUPPORTED) when an element's J is not constant.
template <typename T> static int build_affine(fg_op *op, T **out) {
    int rc;
    T *dst = nullptr;
    if ((rc = alloc_vec(&dst, affine_size<T>(op)))) return rc;
    CK(cudaMemsetAsync(op->d_err, 0, sizeof(int), op->stream));
    switch (op->p) {
    case 1: launch_compress_p<1, T>(op, dst); break;
    case 2: launch_compress_p<2, T>(op, dst); break;
    default: launch_compress_p<3, T>(op, dst); break;
    }
    CK(cudaGetLastError());
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, op->d_err, sizeof(int), cudaMemcpyDeviceToHost, op->stream));
    CK(cudaStreamSynchronize(op->stream));
    if (herr) {
        cudaFree(dst);
        cudaMemsetAsync(op->d_err, 0, sizeof(int), op->stream);
        return fail(FG_UNSUPPORTED, "affine quadrature-data format refused: the mesh has elements "
                                    "whose Jacobian is not constant");
    }
    *out = dst;
    return FG_OK;
}

static int ensure_solver_buffers(fg_op *op) {
    int rc;
    double **v[] = {&op->r, &op->z, &op->pv, &op->ap, &op->xw, &op->bw, &op->cres, &op->cd, &op->ct};
    for (double **b : v)
        if (!*b && (rc = alloc_vec(b, op->Nn))) return rc;
    return FG_OK;
}

static int ensure_dinv(fg_op *op) {
    if (op->have_dinv) return FG_OK;
    int rc;
    if (!op->dinv && (rc = alloc_vec(&op->dinv, op->Nn))) return rc;
    if ((rc = diag_native(op, op->ys, 1))) return rc;
    k_invert_diag<double><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(op->g, op->ys, op->dinv);
    CK(cudaGetLastError());
    op->have_dinv = true;
    return FG_OK;
}

// FP32 copy of the quadrature data (same layout) and the FP32 work vectors.
static int ensure_fp32(fg_op *op) {
    int rc;
    if (!op->qd32) {
        if ((rc = alloc_vec(&op->qd32, op->qsize))) return rc;
        k_to_f32<<<VEC_GRID * 4, VEC_THREADS, 0, op->stream>>>(op->qsize, op->qd, op->qd32);
        CK(cudaGetLastError());
    }
    if (!op->face32 && (rc = alloc_vec(&op->face32, (int64_t)op->g.n_items() * op->g.face_stride())))
        return rc;
    if (op->fmt == 1 && !op->qa32 && (rc = build_affine<float>(op, &op->qa32))) return rc;
    float **v[] = {&op->r32, &op->z32, &op->p32, &op->ap32, &op->e32, &op->b32, &op->cres32,
                   &op->cd32, &op->ct32, &op->xs32, &op->ys32};
    for (float **b : v)
        if (!*b && (rc = alloc_vec(b, op->Nn))) return rc;
    if (!op->st32) {
        CK(cudaMalloc(&op->st32, sizeof(SolverState)));
        CK(cudaMemset(op->st32, 0, sizeof(SolverState)));
        FG_LEGACY_FENCE();
    }
    return FG_OK;
}

static int ensure_dinv32(fg_op *op) {
    int rc;
    if (op->dinv32) return FG_OK;
    if ((rc = ensure_dinv(op))) return rc;
    if ((rc = alloc_vec(&op->dinv32, op->Nn))) return rc;
    k_to_f32<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(op->Nn, op->dinv, op->dinv32);
    CK(cudaGetLastError());
    return FG_OK;
}

static int read_state(fg_op *op, SolverState *h, const SolverState *dev = nullptr) {
    CK(cudaMemcpyAsync(h, dev ? dev : op->st, sizeof(SolverState), cudaMemcpyDeviceToHost, op->stream));
    CK(cudaStreamSynchronize(op->stream));
    return FG_OK;
}

// lambda_max(D^-1 A) by power iteration from the hashed start vector (FP64)
static int estimate_lmax(fg_op *op, int iters, double *out) {
    int rc;
    const int64_t n = op->Nn;
    k_hash_vector<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(op->g, op->cd, op->partials, op->st);
    k_scale_by_rho<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->cd, op->cd, op->st);
    CK(cudaGetLastError());
    for (int it = 0; it < iters; ++it) {
        if ((rc = apply_native(op, op->cd, op->ct, 0, 1, nullptr))) return rc;
        k_dinv_norm<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->ct, op->dinv, op->partials, op->st);
        k_scale_by_rho<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->ct, op->cd, op->st);
        CK(cudaGetLastError());
    }
    SolverState h;
    if ((rc = read_state(op, &h))) return rc;
    *out = h.rho;
    return FG_OK;
}

struct ChebCoef {
    double inv_theta = 0.0;
    std::vector<double> c1, c2;
};
static ChebCoef cheb_coefs(double lmin, double lmax, int k) {
    ChebCoef c;
    const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
    const double sigma = theta / delta;
    double rho = 1.0 / sigma;
    c.inv_theta = 1.0 / theta;
    for (int s = 1; s < k; ++s) {
        const double rn = 1.0 / (2.0 * sigma - rho);
        c.c1.push_back(rn * rho);
        c.c2.push_back(2.0 * rn / delta);
        rho = rn;
    }
    return c;
}

// Buffers of one PCG run in storage precision T.
template <typename T> struct PcgBufs {
    const T *qd;
    T *face;
    const T *dinv;
    T *x, *b, *r, *z, *p, *ap, *cres, *cd, *ct;
    SolverState *st;
};

template <typename T> static T **cheb_dk(fg_op *op);
template <> double **cheb_dk<double>(fg_op *op) { return op->cdk; }
template <> float **cheb_dk<float>(fg_op *op) { return op->cdk32; }

// z = Chebyshev(D^-1 A) r (Saad Alg. 12.1, zero start, k sweeps)
template <typename T>
static int cheb_apply(fg_op *op, const PcgBufs<T> &B, const ChebCoef &cc, const T *r, T *z,
                      const int *skip) {
    const int64_t n = op->Nn;
    const SolverState *sst = skip ? B.st : nullptr;
    const int s = (int)cc.c1.size();
    if (s >= 1 && s <= CHEB_MAXD) {
        // d_k in their own vectors (d_0 = cd), z formed once in the last sweep.
        // The vectors are allocated by the first call, which a solver makes
        // outside graph capture (its first chunk runs directly).
        T **dk = cheb_dk<T>(op);
        for (int k = 1; k < s; ++k)
            if (!dk[k - 1]) {
                int rc = alloc_vec(&dk[k - 1], n);
                if (rc) return rc;
            }
        k_cheb_first_d<T><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, r, B.dinv, B.cres, B.cd,
                                                                    cc.inv_theta, sst);
        CK(cudaGetLastError());
        const T *dprev = B.cd;
        for (int k = 1; k <= s; ++k) {
            int rc = apply_native_t<T>(op, B.qd, B.face, dprev, B.ct, 0, 1, skip);
            if (rc) return rc;
            if (k < s) {
                k_cheb_mid<T><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.ct, B.dinv, B.cres, dprev,
                                                                        dk[k - 1], cc.c1[k - 1],
                                                                        cc.c2[k - 1], sst);
                dprev = dk[k - 1];
            } else {
                ChebSum<T> earlier{};
                earlier.n = s - 1;  // d_0 .. d_{s-2}
                for (int j = 0; j < s - 1; ++j) earlier.d[j] = j == 0 ? B.cd : dk[j - 1];
                k_cheb_last<T><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.ct, B.dinv, B.cres, dprev,
                                                                         earlier, z, cc.c1[k - 1],
                                                                         cc.c2[k - 1], sst);
            }
            CK(cudaGetLastError());
        }
        return FG_OK;
    }
    k_cheb_first<T><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, r, B.dinv, B.cres, B.cd, z,
                                                              cc.inv_theta, sst);
    CK(cudaGetLastError());
    for (size_t s = 0; s < cc.c1.size(); ++s) {
        int rc = apply_native_t<T>(op, B.qd, B.face, B.cd, B.ct, 0, 1, skip);
        if (rc) return rc;
        k_cheb_step<T><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.ct, B.dinv, B.cres, B.cd, z,
                                                                 cc.c1[s], cc.c2[s], sst);
        CK(cudaGetLastError());
    }
    return FG_OK;
}

// PCG on the constrained operator in storage precision T (reductions in FP64),
// par_solver.rs:262-342 semantics.  The state (rtol, atol, max_iter) must be
// loaded into B.st before the call.  x_zero: the initial guess is zero (the
// first residual needs no apply).  Returns the final host copy of the state.
// A chunk of solver iterations (the launches between two host reads of the
// solver state).  The first chunk with a given key is launched directly, which
// also performs every one-time step of the launchers (kernel attributes,
// lazily sized buffers); the second is captured on a private stream into a
// CUDA graph; later ones replay that graph on the handle's stream.  Kernel
// arguments, buffers and the order of launches are the same in every chunk
// of a solve, and all per-iteration state lives in device memory, so a replay
// performs exactly the launches of a direct chunk.
struct ChunkGraph {
    cudaGraphExec_t exec = nullptr;
    int key = -1, iters = 0, seen = 0;
    ChunkGraph() = default;
    ChunkGraph(const ChunkGraph &) = delete;
    ChunkGraph &operator=(const ChunkGraph &) = delete;
    ~ChunkGraph() {
        if (exec) cudaGraphExecDestroy(exec);
    }
};

static int run_chunk(fg_op *op, ChunkGraph &cg, int key, int iters, const std::function<int()> &iteration) {
    auto direct = [&]() -> int {
        for (int k = 0; k < iters; ++k) {
            const int rc = iteration();
            if (rc) return rc;
        }
        return FG_OK;
    };
    if (!op->graphs) return direct();
    if (cg.exec && cg.key == key && cg.iters == iters) {
        CK(cudaGraphLaunch(cg.exec, op->stream));
        return FG_OK;
    }
    if (cg.key != key || cg.iters != iters) {
        if (cg.exec) cudaGraphExecDestroy(cg.exec);
        cg.exec = nullptr;
        cg.key = key;
        cg.iters = iters;
        cg.seen = 0;
    }
    if (cg.seen++ == 0) return direct();
    if (!op->cap_stream) CK(cudaStreamCreateWithFlags(&op->cap_stream, cudaStreamNonBlocking));
    const cudaStream_t saved = op->stream;
    CK(cudaStreamBeginCapture(op->cap_stream, cudaStreamCaptureModeThreadLocal));
    op->stream = op->cap_stream;
    const int rc = direct();
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(op->cap_stream, &graph);
    op->stream = saved;
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (ce != cudaSuccess) return fail(FG_CUDA_ERROR, "graph capture: %s", cudaGetErrorString(ce));
    const cudaError_t ie = cudaGraphInstantiate(&cg.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
        cg.exec = nullptr;
        return fail(FG_CUDA_ERROR, "graph instantiate: %s", cudaGetErrorString(ie));
    }
    CK(cudaGraphLaunch(cg.exec, op->stream));
    return FG_OK;
}

// The vector work of one Jacobi-PCG (or operator-CG) iteration as one
// cooperative launch (k_pcg_fused_jacobi); returns 1 when the device cannot
// hold all VEC_GRID blocks at once (the caller then uses the three kernels).
template <typename T> static int launch_pcg_fused(fg_op *op, const PcgBufs<T> &B, bool *used) {
    *used = false;
    if (!op->fused_pcg) return FG_OK;
    static int fits[64];  // per device: 1 fits, -1 does not, 0 not yet known
    if (op->device < 0 || op->device >= 64) return FG_OK;
    auto kern = k_pcg_fused_jacobi<T>;
    if (!fits[op->device]) {
        int per_sm = 0, sms = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, VEC_THREADS, 0));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, op->device));
        fits[op->device] = per_sm * sms >= VEC_GRID ? 1 : -1;
    }
    if (fits[op->device] < 0) return FG_OK;
    if (!op->bar) {
        CK(cudaMalloc(&op->bar, 2 * sizeof(unsigned)));
        CK(cudaMemset(op->bar, 0, 2 * sizeof(unsigned)));
        FG_LEGACY_FENCE();
    }
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(VEC_GRID);
    lc.blockDim = dim3(VEC_THREADS);
    lc.stream = op->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    T *x = const_cast<T *>(B.x), *r = B.r, *p = B.p, *z = B.z;
    CK(cudaLaunchKernelEx(&lc, kern, op->Nn, x, r, p, (const T *)B.ap, B.dinv, z, op->partials, B.st, op->bar,
                          op->d_err));
    *used = true;
    return FG_OK;
}

template <typename T>
static int pcg_run(fg_op *op, const PcgBufs<T> &B, bool jacobi_like, const ChebCoef *cc,
                   int max_iter, int check_interval, bool x_zero, SolverState *h,
                   int64_t *applies, const std::function<int(int)> &on_chunk = nullptr) {
    int rc;
    const int64_t n = op->Nn;
    const int *skip = &B.st->done;
    const bool cheb = cc != nullptr;
    if (x_zero) {
        CK(cudaMemsetAsync(B.ap, 0, sizeof(T) * n, op->stream));
    } else {
        if ((rc = apply_native_t<T>(op, B.qd, B.face, B.x, B.ap, 0, 1, nullptr))) return rc;
        ++*applies;
    }
    k_pcg_init<T><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.b, B.ap, B.dinv, B.r, B.z, B.p,
                                                            jacobi_like ? 1 : 0, op->partials, B.st);
    CK(cudaGetLastError());
    if (cheb) {
        if ((rc = cheb_apply<T>(op, B, *cc, B.r, B.z, skip))) return rc;
        k_pcg_rz<T><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.r, B.z, op->partials, B.st, 1);
        k_pcg_pupdate<T><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.z, B.p, B.st, 1);
        CK(cudaGetLastError());
    }
    int launched = 0;
    ChunkGraph cg;
    auto iteration = [&]() -> int {
        int r2;
        if ((r2 = apply_native_t<T>(op, B.qd, B.face, B.p, B.ap, 0, 1, skip))) return r2;
        if (!cheb) {
            bool used = false;
            if ((r2 = launch_pcg_fused<T>(op, B, &used))) return r2;
            if (used) return FG_OK;
        }
        k_pcg_pap<T><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.p, B.ap, op->partials, B.st);
        k_pcg_update<T><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(
            n, B.x, B.r, B.p, B.ap, B.dinv, B.z, cheb ? 0 : 1, op->partials, B.st);
        if (cheb) {
            if ((r2 = cheb_apply<T>(op, B, *cc, B.r, B.z, skip))) return r2;
            k_pcg_rz<T><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.r, B.z, op->partials, B.st, 0);
        }
        k_pcg_pupdate<T><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.z, B.p, B.st, 0);
        CK(cudaGetLastError());
        return FG_OK;
    };
    while (launched < max_iter) {
        const int chunk = std::min(check_interval, max_iter - launched);
        if ((rc = run_chunk(op, cg, 0, chunk, iteration))) return rc;
        launched += chunk;
        if ((rc = read_state(op, h, B.st))) return rc;
        if (on_chunk && !h->done && (rc = on_chunk(h->iter))) return rc;
        if (h->done) break;
    }
    if ((rc = read_state(op, h, B.st))) return rc;
    // applies actually executed: one per iteration started, the smoother after the
    // initial residual and after every update that left the solve running
    const int km1 = cheb ? (int)cc->c1.size() : 0;
    const bool stopped_by_update = h->converged || (!h->breakdown && h->iter >= max_iter);
    if (!(h->iter == 0 && h->done && !h->breakdown)) *applies += km1;
    *applies += h->iter + (h->breakdown ? 1 : 0);
    *applies += (int64_t)km1 * (h->iter - (stopped_by_update ? 1 : 0));
    return FG_OK;
}

// ---- learned coarse correction inside the preconditioner -------------------
// The DOF lattice (NI, NJ, NK) -- uniform for equispaced nodes of any order --
// is coarsened nn_levels = L times (vertex-centred) to the network volume.
// rcoarse = R^L r, s = rms(rcoarse), network input (rcoarse / s, R^L log kappa),
// correction c = s 8^L P^L n (zero on essential DOFs).  With P^T = 8 R per
// level the Galerkin optimum is n = (P^T A P)^{-1} (R^L r / s), whose scale
// does not depend on the fine resolution.
static Vol nn_vol(const fg_op *op, int level) {
    Vol v{1, op->g.NK, op->g.NJ, op->g.NI};
    for (int l = 0; l < level; ++l) v = Vol{1, (v.Z + 1) / 2, (v.Y + 1) / 2, (v.X + 1) / 2};
    return v;
}
static Vol nn_coarse_vol(const fg_op *op) { return nn_vol(op, op->nn_levels); }
static double nn_mult(const fg_op *op) { return std::ldexp(1.0, 3 * op->nn_levels); }

// network-level coarse field of a fine native vector r (FP32, into dst)
template <typename T> static int nn_restrict(fg_op *op, const T *r, float *dst) {
    Grid g = op->g;
    const int L = op->nn_levels;
    int blocks;
    Vol v1 = nn_vol(op, 1);
    grid_launch(v1.nvox(), blocks);
    fe_restrict_kernel<T><<<blocks, 256, 0, op->stream>>>(g, r, L == 1 ? dst : op->nn_tmp[0], v1);
    for (int l = 2; l <= L; ++l) {
        const Vol vf = nn_vol(op, l - 1), vc = nn_vol(op, l);
        grid_launch(vc.nvox(), blocks);
        restrict_f32_kernel<<<blocks, 256, 0, op->stream>>>(op->nn_tmp[l - 2], vf, l == L ? dst : op->nn_tmp[l - 1],
                                                            vc, 1.f);
    }
    CK(cudaGetLastError());
    return FG_OK;
}

// level-1 FP32 field P^(L-1) oc of the network-level field oc (on op->stream)
static const float *nn_prolong_to_level1(fg_op *op, const float *oc) {
    const float *f = oc;
    for (int l = op->nn_levels - 1; l >= 1; --l) {
        const Vol vc = nn_vol(op, l + 1), vf = nn_vol(op, l);
        int blocks;
        grid_launch(vf.nvox(), blocks);
        prolong_f32_kernel<<<blocks, 256, 0, op->stream>>>(f, vc, op->nn_tmp[l - 1], vf);
        f = op->nn_tmp[l - 1];
    }
    return f;
}

// fine native z (+)= scale[0] * mult * P f1 (level-1 FP32 field f1)
template <typename T>
static int nn_fe_prolong(fg_op *op, const float *f1, T *z, const double *scale, double mult, int accumulate) {
    Grid g = op->g;
    g.ess = op->ess_tags;
    if (g.NJ > 65535 || g.NK > 65535) return fail(FG_UNSUPPORTED, "prolongation grid: more than 65535 DOF rows");
    const int pairs = g.NIp / 2;
    const int bd = std::min(256, (pairs + 31) / 32 * 32);
    const dim3 grid((pairs + bd - 1) / bd, g.NJ, g.NK);
    fe_prolong_f32_kernel<T><<<grid, bd, 0, op->stream>>>(g, f1, nn_vol(op, 1), z, scale, mult, accumulate);
    CK(cudaGetLastError());
    return FG_OK;
}

// fine native z (+)= scale[0] * mult * P^L (network-level FP32 field oc)
template <typename T>
static int nn_prolong(fg_op *op, const float *oc, T *z, const double *scale, double mult, int accumulate) {
    const float *f1 = nn_prolong_to_level1(op, oc);
    CK(cudaGetLastError());
    return nn_fe_prolong<T>(op, f1, z, scale, mult, accumulate);
}

// z += s 8^L P^L(UNet(R^L r / s, R^L log kappa)),  s = rms(R^L r), in two
// halves around the Chebyshev smoother, which reads the same r:
//   nn_begin: restriction, network and the coarse prolongations, issued on a
//             high-priority side stream forked from op->stream (event), so the
//             small latency-bound network kernels run beside the smoother's
//             bandwidth-bound applies;
//   nn_end:   op->stream waits for the side stream, then adds the last
//             prolongation into z (after the smoother has written z).
// The fork and join are events, so a chunk captured into a CUDA graph records
// them as graph edges.  No buffer is shared between the two streams except r
// (read by both) and the network's own buffers (side stream only).
template <typename T> static int nn_begin(fg_op *op, const T *r, const float **f1) {
    fg_unet *u = op->nn;
    const Vol Vc = nn_coarse_vol(op);
    int rc;
    if ((rc = unet_ensure_bufs(u, 1, Vc.Z, Vc.Y, Vc.X))) return rc;
    const cudaStream_t main = op->stream;
    struct Restore { fg_op *o; cudaStream_t s; ~Restore() { o->stream = s; } } restore{op, main};
    if (op->nn_overlap) {
        if (!op->nn_stream) {
            int lo = 0, hi = 0;
            CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            CK(cudaStreamCreateWithPriority(&op->nn_stream, cudaStreamNonBlocking, hi));
            CK(cudaEventCreateWithFlags(&op->nn_ev_r, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&op->nn_ev_n, cudaEventDisableTiming));
        }
        CK(cudaEventRecord(op->nn_ev_r, main));
        CK(cudaStreamWaitEvent(op->nn_stream, op->nn_ev_r, 0));
        op->stream = op->nn_stream;
    }
    u->stream = op->stream;
    u->err = op->d_err;
    const int64_t nv = Vc.nvox();
    int blocks;
    grid_launch(nv, blocks);
    if ((rc = nn_restrict<T>(op, r, op->nn_rc))) return rc;
    rms_kernel<<<1, 1024, 0, op->stream>>>(op->nn_rc, nv, op->nn_scale);
    pack_input_kernel<<<blocks, 256, 0, op->stream>>>(op->nn_rc, op->nn_lk, nv, op->nn_scale,
                                                      TView{u->buf.x0, 2, 0});
    CK(cudaGetLastError());
    if ((rc = unet_forward(u))) return rc;
    out0_to_f32_kernel<<<blocks, 256, 0, op->stream>>>(TView{u->buf.out, 8, 0}, nv, op->nn_oc);
    *f1 = nn_prolong_to_level1(op, op->nn_oc);
    CK(cudaGetLastError());
    if (op->nn_overlap) CK(cudaEventRecord(op->nn_ev_n, op->stream));
    return FG_OK;
}

template <typename T> static int nn_end(fg_op *op, const float *f1, T *z) {
    if (op->nn_overlap) CK(cudaStreamWaitEvent(op->stream, op->nn_ev_n, 0));
    return nn_fe_prolong<T>(op, f1, z, op->nn_scale, nn_mult(op), 1);
}

// Device time of one preconditioned iteration without and with the learned
// correction (the operator apply, then the Chebyshev smoother, the network
// beside it), in storage precision T, on the solve's own buffers: r holds the
// right-hand side (the network sees a residual-like input) and p a copy of it.
// Three timed repetitions after one warm-up each, CUDA events on the handle's
// stream.  Used before the timed solve to decide whether the network pays.
template <typename T>
static int nn_iteration_times(fg_op *op, const PcgBufs<T> &B, const ChebCoef &cc, T *r, T *z, T *p, T *ap,
                              double *plain_ms, double *learned_ms) {
    auto plain = [&]() -> int {
        int rc = apply_native_t<T>(op, B.qd, B.face, p, ap, 0, 1, nullptr);
        return rc ? rc : cheb_apply<T>(op, B, cc, r, z, nullptr);
    };
    auto learned = [&]() -> int {
        const float *f1 = nullptr;
        int rc = apply_native_t<T>(op, B.qd, B.face, p, ap, 0, 1, nullptr);
        if (!rc) rc = nn_begin<T>(op, r, &f1);
        if (!rc) rc = cheb_apply<T>(op, B, cc, r, z, nullptr);
        return rc ? rc : nn_end<T>(op, f1, z);
    };
    auto timed = [&](const std::function<int()> &fn, double *ms) -> int {
        int rc = fn();
        if (rc) return rc;
        CK(cudaEventRecord(op->ev0, op->stream));
        for (int k = 0; k < 3; ++k)
            if ((rc = fn())) return rc;
        CK(cudaEventRecord(op->ev1, op->stream));
        CK(cudaEventSynchronize(op->ev1));
        float m = 0.f;
        CK(cudaEventElapsedTime(&m, op->ev0, op->ev1));
        *ms = m / 3.0;
        return FG_OK;
    };
    int rc = timed(plain, plain_ms);
    return rc ? rc : timed(learned, learned_ms);
}

// Flexible CG (FCG(1), Notay) with z = Chebyshev(r) [+ learned correction];
// once `budget` iterations pass without convergence the learned term is
// dropped and the solve continues as plain Chebyshev-preconditioned CG from
// the current iterate (the fallback).  FP64 storage.
static int fcg_nn_run(fg_op *op, const PcgBufs<double> &B, const ChebCoef &cc, int max_iter,
                      int check_interval, int budget, SolverState *h, int64_t *applies,
                      int *fell_back) {
    int rc;
    const int64_t n = op->Nn;
    const int *skip = &B.st->done;
    bool nn_on = op->nn != nullptr;
    *fell_back = 0;
    if ((rc = apply_native_t<double>(op, B.qd, B.face, B.x, B.ap, 0, 1, nullptr))) return rc;
    ++*applies;
    k_pcg_init<double><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.b, B.ap, B.dinv, B.r, B.z, B.p,
                                                                 0, op->partials, B.st);
    auto direction = [&](int init) -> int {
        const float *f1 = nullptr;
        int r2;
        if (nn_on && (r2 = nn_begin<double>(op, B.r, &f1))) return r2;
        if ((r2 = cheb_apply<double>(op, B, cc, B.r, B.z, skip))) return r2;
        if (nn_on && (r2 = nn_end<double>(op, f1, B.z))) return r2;
        k_fcg_zap<double><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.z, B.ap, op->partials, B.st, init);
        k_fcg_pupdate_pr<double><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.z, B.p, B.r, op->partials,
                                                                            B.st, init);
        CK(cudaGetLastError());
        return FG_OK;
    };
    if ((rc = direction(1))) return rc;
    int launched = 0;
    ChunkGraph cg;
    auto iteration = [&]() -> int {
        int r2;
        if ((r2 = apply_native_t<double>(op, B.qd, B.face, B.p, B.ap, 0, 1, skip))) return r2;
        k_pcg_pap<double><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.p, B.ap, op->partials, B.st);
        k_pcg_update<double><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, B.x, B.r, B.p, B.ap, B.dinv,
                                                                       B.z, 0, op->partials, B.st);
        return direction(0);
    };
    while (launched < max_iter) {
        const int chunk = std::min(check_interval, max_iter - launched);
        if ((rc = run_chunk(op, cg, nn_on ? 1 : 0, chunk, iteration))) return rc;
        launched += chunk;
        if ((rc = read_state(op, h, B.st))) return rc;
        if (h->done) break;
        if (nn_on && budget > 0 && h->iter >= budget) {
            nn_on = false;
            *fell_back = 1;
        }
    }
    if ((rc = read_state(op, h, B.st))) return rc;
    const int km1 = (int)cc.c1.size();
    *applies += (int64_t)(h->iter + 1) * (1 + km1);
    return FG_OK;
}

static void set_state(fg_op *op, SolverState *dst, double rtol, double atol, int max_iter, int cgop = 0) {
    SolverState h{};
    h.rtol = rtol;
    h.atol = atol;
    h.max_iter = max_iter;
    h.cgop = cgop;
    cudaMemcpyAsync(dst, &h, sizeof h, cudaMemcpyHostToDevice, op->stream);
}

extern "C" {

static int to_native32(fg_op *op, float *dst, const float *src, int mem) {
    return to_native_t<float>(op, dst, src, mem);
}
static int from_native32(fg_op *op, float *dst, const float *src, int mem) {
    return from_native_t<float>(op, dst, src, mem);
}

FG_API int fg_op_set_qdata_format(fg_op *op, int format) {
    if (format != FG_QDATA_FULL) FG_NEED_BOX(op, "the affine quadrature-data format");
    if (!op) return fail(FG_INVALID_ARGUMENT, "NULL op");
    if (format != FG_QDATA_FULL && format != FG_QDATA_AFFINE)
        return fail(FG_INVALID_ARGUMENT, "bad quadrature-data format %d", format);
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    if (format == FG_QDATA_AFFINE) {
        int rc;
        if (!op->qa64 && (rc = build_affine<double>(op, &op->qa64))) return rc;
        if (op->qd32 && !op->qa32 && (rc = build_affine<float>(op, &op->qa32))) return rc;
    }
    op->fmt = format;
    return FG_OK;
}

FG_API int fg_op_apply_f32(fg_op *op, const float *x, float *y, int accumulate, int constrained,
                           int mem) {
    if (!op || !x || !y) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (mem != FG_HOST && mem != FG_DEVICE) return fail(FG_INVALID_ARGUMENT, "bad mem %d", mem);
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    int rc;
    if ((rc = ensure_fp32(op))) return rc;
    if ((rc = to_native32(op, op->xs32, x, mem))) return rc;
    if (accumulate && (rc = to_native32(op, op->ys32, y, mem))) return rc;
    if ((rc = apply_native_t<float>(op, op->qd32, op->face32, op->xs32, op->ys32, accumulate,
                                    constrained, nullptr)))
        return rc;
    if ((rc = from_native32(op, y, op->ys32, mem))) return rc;
    return check_device_error(op);
}

FG_API int fg_op_apply_native_f32(fg_op *op, const float *x, float *y, int accumulate,
                                  int constrained) {
    if (!op || !x || !y) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (x == y) return fail(FG_INVALID_ARGUMENT, "x and y must not alias");
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    int rc;
    if ((rc = ensure_fp32(op))) return rc;
    return apply_native_t<float>(op, op->qd32, op->face32, x, y, accumulate, constrained, nullptr);
}

static int validate_cfg(fg_cfg &cfg) {
    if (cfg.max_iter < 0) return fail(FG_INVALID_ARGUMENT, "max_iter < 0");
    if (cfg.precision != FG_FP64 && cfg.precision != FG_FP32_IR)
        return fail(FG_UNSUPPORTED, "precision %d not available", cfg.precision);
    if (cfg.precond < 0 || cfg.precond > 3) return fail(FG_INVALID_ARGUMENT, "bad precond");
    if ((cfg.precond == FG_PC_CHEBYSHEV || cfg.precond == FG_PC_CHEB_NN) && cfg.cheb_degree < 1)
        return fail(FG_INVALID_ARGUMENT, "cheb_degree must be >= 1");
    if (cfg.check_interval < 1) cfg.check_interval = 10;
    return FG_OK;
}

// PCG on op->bw (right-hand side) from op->xw (initial guess), both native and
// resident; the solution is left in op->xw.  The caller holds op->mu.
static int pcg_core(fg_op *op, const fg_cfg &cfg, fg_result *res) {
    const bool learned = cfg.precond == FG_PC_CHEB_NN;
    if (learned && (!op->nn || !op->nn_lk))
        return fail(FG_INVALID_ARGUMENT, "FG_PC_CHEB_NN needs fg_op_set_nodal_kappa and fg_op_attach_unet");
    const bool cheb = cfg.precond == FG_PC_CHEBYSHEV || learned;
    int fell_back = 0;
    const bool ir = cfg.precision == FG_FP32_IR;
    int rc;
    if ((rc = ensure_solver_buffers(op))) return rc;
    const double *dinv_use = op->dinv;
    if (cfg.precond == FG_PC_NONE) {
        // operator CG: z = r, i.e. Jacobi with an identity diagonal (pads zero)
        if (!op->ones) {
            if ((rc = alloc_vec(&op->ones, op->Nn))) return rc;
            k_invert_diag<double><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(op->g, op->ones, op->ones);
            CK(cudaGetLastError());
        }
        dinv_use = op->ones;
    } else if ((rc = ensure_dinv(op))) {
        return rc;
    } else {
        dinv_use = op->dinv;
    }
    double lmax = 0.0, lmin = 0.0;
    if (cheb) {
        if (cfg.lmax > 0) {
            lmax = cfg.lmax;
        } else {
            if (!op->have_lmax) {
                if ((rc = estimate_lmax(op, cfg.power_iters > 0 ? cfg.power_iters : 20, &op->lmax_est)))
                    return rc;
                op->have_lmax = true;
            }
            lmax = (cfg.lmax_safety > 0 ? cfg.lmax_safety : 1.1) * op->lmax_est;
        }
        lmin = lmax / (cfg.lmin_ratio > 0 ? cfg.lmin_ratio : 30.0);
    }
    const ChebCoef cc = cheb ? cheb_coefs(lmin, lmax, cfg.cheb_degree) : ChebCoef{};
    const int64_t n = op->Nn;
    int64_t applies = 0;
    SolverState h{};
    int outer = 1, inner_total = 0, status = FG_OK;
    // one-time preparation (FP32 copies, network buffers) outside the timed solve
    if (ir) {
        if ((rc = ensure_fp32(op))) return rc;
        if (cfg.precond != FG_PC_NONE && (rc = ensure_dinv32(op))) return rc;
    }
    if (learned) {
        const Vol Vc = nn_coarse_vol(op);
        if ((rc = unet_ensure_bufs(op->nn, 1, Vc.Z, Vc.Y, Vc.X))) return rc;
    }
    // Whether the network pays: with the plain iteration count (nn_budget) and
    // the network's expected iteration ratio (nn_iter_ratio) given, the learned
    // solve is predicted to take ratio * budget iterations of the learned cost
    // against budget iterations of the plain cost; the per-iteration costs are
    // measured once per handle, format and degree (outside the timed solve).
    // When the prediction is not faster the solve runs as plain Chebyshev-PCG
    // from the start (nn_fallback = 2).
    bool use_nn = learned;
    if (learned && cfg.nn_budget > 0 && cfg.nn_iter_ratio > 0.0) {
        const int deg = cfg.cheb_degree;
        const fg_op::NnTimes *t = nullptr;
        for (const auto &e : op->nn_times)
            if (e.ir == (int)ir && e.fmt == op->fmt && e.degree == deg) t = &e;
        if (!t) {
            fg_op::NnTimes e{(int)ir, op->fmt, deg, 0.0, 0.0};
            set_state(op, op->st, cfg.rtol, cfg.atol, cfg.max_iter);
            if (!ir) {
                PcgBufs<double> B{op->qd, op->face, dinv_use, op->xw, op->bw, op->r, op->z, op->pv,
                                  op->ap, op->cres, op->cd, op->ct, op->st};
                CK(cudaMemcpyAsync(op->r, op->bw, sizeof(double) * n, cudaMemcpyDeviceToDevice, op->stream));
                CK(cudaMemcpyAsync(op->pv, op->bw, sizeof(double) * n, cudaMemcpyDeviceToDevice, op->stream));
                rc = nn_iteration_times<double>(op, B, cc, op->r, op->z, op->pv, op->ap, &e.plain_ms,
                                                &e.learned_ms);
            } else {
                PcgBufs<float> B{op->qd32, op->face32, op->dinv32, op->e32, nullptr, op->r32, op->z32, op->p32,
                                 op->ap32, op->cres32, op->cd32, op->ct32, op->st};
                k_to_f32<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->bw, op->r32);
                k_to_f32<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->bw, op->p32);
                CK(cudaGetLastError());
                rc = nn_iteration_times<float>(op, B, cc, op->r32, op->z32, op->p32, op->ap32, &e.plain_ms,
                                               &e.learned_ms);
            }
            if (rc) return rc;
            op->nn_times.push_back(e);
            t = &op->nn_times.back();
        }
        if (cfg.nn_iter_ratio * t->learned_ms >= t->plain_ms) {
            use_nn = false;
            fell_back = 2;
        }
    }
    CK(cudaStreamSynchronize(op->stream));
    CK(cudaEventRecord(op->ev0, op->stream));
    if (!ir) {
        PcgBufs<double> B{op->qd, op->face, dinv_use, op->xw, op->bw, op->r, op->z, op->pv,
                          op->ap, op->cres, op->cd, op->ct, op->st};
        // FG_PC_NONE is the operator CG of solve_cg_operator, with its stopping rule
        set_state(op, op->st, cfg.rtol, cfg.atol, cfg.max_iter, cfg.precond == FG_PC_NONE ? 1 : 0);
        if (learned && use_nn) {
            if ((rc = fcg_nn_run(op, B, cc, cfg.max_iter, cfg.check_interval, cfg.nn_budget, &h, &applies,
                                 &fell_back)))
                return rc;
        } else if ((rc = pcg_run<double>(op, B, !cheb, cheb ? &cc : nullptr, cfg.max_iter,
                                         cfg.check_interval, false, &h, &applies)))
            return rc;
        inner_total = h.iter;
        status = h.converged ? FG_OK : (h.breakdown ? FG_BREAKDOWN : FG_CONVERGENCE_FAILED);
    } else {
        // Mixed-precision PCG with reliable updates: FP32 applies, smoother and
        // iterates; FP64 solution, true residual and dot products.
        if ((rc = ensure_fp32(op))) return rc;
        const float *dinv32 = nullptr;
        if (cfg.precond == FG_PC_NONE) {
            if (!op->dinv32 && (rc = alloc_vec(&op->dinv32, op->Nn))) return rc;
            k_to_f32<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->ones, op->dinv32);
            dinv32 = op->dinv32;
        } else {
            if ((rc = ensure_dinv32(op))) return rc;
            dinv32 = op->dinv32;
        }
        PcgBufs<float> B{op->qd32, op->face32, dinv32, op->e32, nullptr, op->r32, op->z32, op->p32,
                         op->ap32, op->cres32, op->cd32, op->ct32, op->st};
        SolverState h0{};
        h0.rtol = cfg.rtol;
        h0.atol = cfg.atol;
        h0.max_iter = cfg.max_iter;
        h0.delta = (cfg.inner_rtol > 0 && cfg.inner_rtol < 1) ? cfg.inner_rtol : 0.1;
        CK(cudaMemcpyAsync(op->st, &h0, sizeof h0, cudaMemcpyHostToDevice, op->stream));
        CK(cudaMemsetAsync(op->e32, 0, sizeof(float) * n, op->stream));
        const int *done = &op->st->done;
        const int *skip_rel = &op->st->skip_rel;
        // r = b - A x (FP64), r_lo = r
        if ((rc = apply_native(op, op->xw, op->ap, 0, 1, nullptr))) return rc;
        ++applies;
        k_rel_residual<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->bw, op->ap, op->r32,
                                                                 op->partials, op->st, 1);
        // z = M r_lo ; p = z ; rz
        bool nn_on = learned && use_nn;
        auto precond = [&](int init) -> int {
            if (learned && use_nn) {  // flexible directions: z = Chebyshev(r) [+ learned correction]
                const float *f1 = nullptr;
                int rc2;
                if (nn_on && (rc2 = nn_begin<float>(op, op->r32, &f1))) return rc2;
                if ((rc2 = cheb_apply<float>(op, B, cc, op->r32, op->z32, done))) return rc2;
                if (nn_on && (rc2 = nn_end<float>(op, f1, op->z32))) return rc2;
                k_fcg_zap<float><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->z32, op->ap32, op->partials,
                                                                           op->st, init);
                k_fcg_pupdate_pr<float><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->z32, op->p32, op->r32,
                                                                                   op->partials, op->st, init);
                CK(cudaGetLastError());
                return FG_OK;
            }
            if (cheb) {
                int rc2 = cheb_apply<float>(op, B, cc, op->r32, op->z32, done);
                if (rc2) return rc2;
                k_pcg_rz<float><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->r32, op->z32,
                                                                          op->partials, op->st, init);
            } else {
                k_jacobi_rz<float><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->r32, dinv32, op->z32,
                                                                             op->partials, op->st, init);
            }
            k_pcg_pupdate<float><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->z32, op->p32, op->st, init);
            CK(cudaGetLastError());
            return FG_OK;
        };
        if ((rc = precond(1))) return rc;
        int launched = 0;
        ChunkGraph cg;
        auto iteration = [&]() -> int {
            int r2;
            if ((r2 = apply_native_t<float>(op, op->qd32, op->face32, op->p32, op->ap32, 0, 1, done))) return r2;
            k_pcg_pap<float><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->p32, op->ap32, op->partials, op->st);
            k_rel_step<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->e32, op->r32, op->p32, op->ap32,
                                                                 op->partials, op->st);
            // reliable update (kernels return at once unless triggered)
            k_rel_xupdate<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->xw, op->e32, op->st);
            if ((r2 = apply_native(op, op->xw, op->ap, 0, 1, skip_rel))) return r2;
            k_rel_residual<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->bw, op->ap, op->r32, op->partials,
                                                                     op->st, 0);
            return precond(0);
        };
        while (launched < cfg.max_iter) {
            const int chunk = std::min(cfg.check_interval, cfg.max_iter - launched);
            if ((rc = run_chunk(op, cg, nn_on ? 1 : 0, chunk, iteration))) return rc;
            launched += chunk;
            if ((rc = read_state(op, &h))) return rc;
            if (h.done) break;
            if (nn_on && cfg.nn_budget > 0 && h.iter >= cfg.nn_budget) {
                nn_on = false;
                fell_back = 1;
            }
        }
        if ((rc = read_state(op, &h))) return rc;
        inner_total = h.iter;
        outer = (int)h.tmp[1];  // reliable (FP64 residual-replacing) updates
        status = h.converged ? FG_OK : (h.breakdown ? FG_BREAKDOWN : FG_CONVERGENCE_FAILED);
        const int km1 = cheb ? (int)cc.c1.size() : 0;
        applies += (int64_t)h.iter * (1 + km1) + km1;
    }
    CK(cudaEventRecord(op->ev1, op->stream));
    // true residual in FP64
    if ((rc = apply_native(op, op->xw, op->ap, 0, 1, nullptr))) return rc;
    k_true_residual<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->bw, op->ap, op->partials, op->st);
    CK(cudaGetLastError());
    SolverState h2;
    if ((rc = read_state(op, &h2))) return rc;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, op->ev0, op->ev1);
    if ((rc = check_device_error(op))) return rc;
    const bool conv = status == FG_OK;
    if (res) {
        res->converged = conv;
        res->iterations = conv ? inner_total : (status == FG_BREAKDOWN ? inner_total : cfg.max_iter);
        res->final_residual = ir ? h.res : h.res;
        res->true_residual = h2.tmp[0];
        res->status = status;
        res->outer_iterations = outer;
        res->applies = applies;
        res->lmax = lmax;
        res->solve_ms = ms;
        res->nn_fallback = fell_back;
    }
    if (cfg.print_level >= 1)
        fprintf(stderr, "fg_pcg: %s after %d iterations (%d outer), residual %.3e (true %.3e)\n",
                conv ? "converged" : "not converged", inner_total, outer, h.res, h2.tmp[0]);
    if (status == FG_OK) t_last_status = FG_OK;
    else if (status == FG_BREAKDOWN) fail(status, "CG breakdown: p^T A p is near zero");
    else fail(status, "solver did not converge in %d iterations (residual = %.3e)", cfg.max_iter, h.res);
    return status;
}

// ---------------------------------------------------------------------------
// Batched mixed-precision PCG (many independent operators in one launch per
// phase).  Helpers live outside extern "C" (templates).
// ---------------------------------------------------------------------------
}  // extern "C"

template <int P, typename T, int FMT>
static int encode_xmap_t(const Grid &g, const T *x, CUtensorMap *tmap) {
    using C = KC<P, T>;
    constexpr int S = FMT == 0 ? C::S : affine_stages<P, T>();
    using SM = ApplySmem<P, T, C::WY, S, 1>;
    cuuint64_t gdim[3] = {(cuuint64_t)g.NI, (cuuint64_t)g.NJ, (cuuint64_t)g.NK};
    cuuint64_t gstr[2] = {(cuuint64_t)g.NIp * sizeof(T), (cuuint64_t)g.NIp * g.NJ * sizeof(T)};
    cuuint32_t box[3] = {(cuuint32_t)SM::XW, (cuuint32_t)SM::RY, (cuuint32_t)(P + 1)};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult cr = g_encode(tmap, TmapType<T>::v, 3, const_cast<T *>(x), gdim, gstr, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return fail(FG_CUDA_ERROR, "cuTensorMapEncodeTiled failed (%d)", (int)cr);
    return FG_OK;
}
template <typename T> static int encode_xmap(fg_op *op, const T *x, CUtensorMap *tmap) {
    switch (op->p) {
    case 1: return encode_xmap_t<1, T, 0>(op->g, x, tmap);
    case 2: return encode_xmap_t<2, T, 0>(op->g, x, tmap);
    default: return encode_xmap_t<3, T, 0>(op->g, x, tmap);
    }
}

struct BatchGroup {
    int p, kind, fmt;
    std::vector<int> inst;
    int2 *bmap = nullptr;
    int nblocks = 0;
};

template <int P, int OPK, typename T, int FMT>
static int launch_batched_t(cudaStream_t st, const BatchGroup &G, const ApplyArgs<T> *args,
                            const CUtensorMap *tm, int nslots, int slot) {
    using C = KC<P, T>;
    constexpr int S = FMT == 0 ? C::S : affine_stages<P, T>();
    using SM = ApplySmem<P, T, C::WY, S, stage_elems<P, OPK, FMT>() / 32>;
    auto kern = pa_apply_batched_kernel<P, OPK, T, C::WY, S, apply_minb<P, T, FMT, C::MINB>(), FMT>;
    static std::atomic<bool> attr_set[64];
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(FG_CUDA_ERROR, "device id %d out of range", dev);
    if (!attr_set[dev].load(std::memory_order_acquire)) {  // set once, before any capture (see fg_batch_pcg)
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SM::bytes));
        attr_set[dev].store(true, std::memory_order_release);
    }
    if (!args) return FG_OK;  // attribute preparation only
    BatchApply<T> B{args, tm, G.bmap, nslots, slot};
    kern<<<G.nblocks, C::WY * 32, SM::bytes, st>>>(B);
    CK(cudaGetLastError());
    return FG_OK;
}
template <typename T>
static int launch_batched(cudaStream_t st, const BatchGroup &G, const ApplyArgs<T> *args,
                          const CUtensorMap *tm, int nslots, int slot) {
#define FG_BL(P_, K_, F_) \
    if (G.p == P_ && G.kind == K_ && G.fmt == F_) return launch_batched_t<P_, K_, T, F_>(st, G, args, tm, nslots, slot);
    FG_BL(1, 1, 0) FG_BL(1, 2, 0) FG_BL(1, 3, 0) FG_BL(2, 1, 0) FG_BL(2, 2, 0) FG_BL(2, 3, 0)
    FG_BL(3, 1, 0) FG_BL(3, 2, 0) FG_BL(3, 3, 0)
    FG_BL(1, 1, 1) FG_BL(1, 2, 1) FG_BL(1, 3, 1) FG_BL(2, 1, 1) FG_BL(2, 2, 1) FG_BL(2, 3, 1)
    FG_BL(3, 1, 1) FG_BL(3, 2, 1) FG_BL(3, 3, 1)
#undef FG_BL
    return fail(FG_UNSUPPORTED, "no batched kernel for this order/kind/format");
}

template <typename T> static int dev_upload(T **dst, const std::vector<T> &v) {
    CK(cudaMalloc(dst, sizeof(T) * std::max<size_t>(v.size(), 1)));
    CK(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    FG_LEGACY_FENCE();
    return FG_OK;
}

// ---- tile shape: items of 32 x WY x TZ elements -----------------------------
template <int P, int OPK> static int relayout_t(fg_op *op, const Grid &gn, double *dst) {
    const int64_t total = (int64_t)op->g.nx * op->g.ny * op->g.nz * (P + 1) * (P + 1) * (P + 1);
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
    qdata_relayout_kernel<P, OPK><<<blocks, 256, 0, op->stream>>>(op->g, gn, op->qd, dst);
    CK(cudaGetLastError());
    return FG_OK;
}
template <int P> static int relayout_p(fg_op *op, const Grid &gn, double **dst, int64_t *size) {
    switch (op->kind) {
    case FG_MASS: *size = qd_size<P, 1>(gn); break;
    case FG_DIFF: *size = qd_size<P, 2>(gn); break;
    default: *size = qd_size<P, 3>(gn); break;
    }
    int rc;
    if ((rc = alloc_vec(dst, *size))) return rc;
    switch (op->kind) {
    case FG_MASS: return relayout_t<P, 1>(op, gn, *dst);
    case FG_DIFF: return relayout_t<P, 2>(op, gn, *dst);
    default: return relayout_t<P, 3>(op, gn, *dst);
    }
}

// Move the operator to items of TZ = tz layers (caller holds op->mu): the
// full quadrature data is re-laid out on the device, the face slots are
// re-sized, and the FP32 / affine copies are dropped and rebuilt from the new
// layout on next use (the affine FP64 copy at once if it is in use).
static int set_tile_locked(fg_op *op, int tz) {
    if (tz == op->g.TZ) return FG_OK;
    Grid gn = op->g;
    gn.TZ = tz;
    gn.ntz = (gn.nz + tz - 1) / tz;
    double *nq = nullptr, *nface = nullptr;
    int64_t nsize = 0;
    int rc;
    switch (op->p) {
    case 1: rc = relayout_p<1>(op, gn, &nq, &nsize); break;
    case 2: rc = relayout_p<2>(op, gn, &nq, &nsize); break;
    default: rc = relayout_p<3>(op, gn, &nq, &nsize); break;
    }
    if (!rc) rc = alloc_vec(&nface, (int64_t)gn.n_items() * gn.face_stride());
    if (!rc && cudaStreamSynchronize(op->stream) != cudaSuccess)
        rc = fail(FG_CUDA_ERROR, "quadrature-data re-layout failed: %s", cudaGetErrorString(cudaGetLastError()));
    if (rc) {
        if (nq) cudaFree(nq);
        if (nface) cudaFree(nface);
        return rc;
    }
    cudaFree(op->qd);
    cudaFree(op->face);
    float **f32[] = {&op->qd32, &op->face32, &op->qa32};
    for (float **b : f32)
        if (*b) { cudaFree(*b); *b = nullptr; }
    if (op->qa64) { cudaFree(op->qa64); op->qa64 = nullptr; }
    op->qd = nq;
    op->face = nface;
    op->qsize = nsize;
    op->g = gn;
    if (op->fmt == 1 && (rc = build_affine<double>(op, &op->qa64))) return rc;
    return FG_OK;
}

// batched launches over a set of instances: block map with the instances
// holding the most items first (fewer idle SMs at the end of a launch)
static std::vector<int2> largest_first_bmap(fg_op *const *ops, const std::vector<int> &inst,
                                            const std::vector<int> &slot_of) {
    std::vector<int> order(inst.size());
    for (size_t k = 0; k < inst.size(); ++k) order[k] = (int)k;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return ops[inst[a]]->g.n_items() > ops[inst[b]]->g.n_items();
    });
    std::vector<int2> m;
    for (int k : order)
        for (int it = 0; it < ops[inst[k]]->g.n_items(); ++it) m.push_back(make_int2(slot_of[k], it));
    return m;
}

static const int kTuneTZ[FG_TUNE_CANDIDATES] = {1, 2, 4, 8, 16};

// time `reps` batched FP32 applies (apply + fix-up) of the instances `inst`
// in their current tile shapes; microseconds per apply
static int time_batched_apply(fg_op *const *ops, const std::vector<int> &inst, cudaStream_t bs, int reps,
                              double *us) {
    const int k = (int)inst.size();
    std::vector<ApplyArgs<float>> a(k);
    std::vector<CUtensorMap> t(k);
    std::vector<FixArgs<float>> f(k);
    std::vector<int> slot(k);
    int rc;
    for (int j = 0; j < k; ++j) {
        fg_op *o = ops[inst[j]];
        if ((rc = ensure_fp32(o))) return rc;
        Grid g = o->g;
        g.ess = o->ess_tags;
        a[j] = ApplyArgs<float>{g, qdata_of<float>(o), o->ap32, o->face32, 0, o->d_err, nullptr};
        if ((rc = encode_xmap<float>(o, o->p32, &t[j]))) return rc;
        f[j] = FixArgs<float>{g, o->ap32, o->face32, nullptr};
        slot[j] = j;
        CK(cudaStreamSynchronize(o->stream));
    }
    fg_op *o0 = ops[inst[0]];
    BatchGroup G{o0->p, o0->kind, o0->fmt, {}};
    const std::vector<int2> m = largest_first_bmap(ops, inst, slot);
    G.nblocks = (int)m.size();
    ApplyArgs<float> *d_a = nullptr;
    CUtensorMap *d_t = nullptr;
    FixArgs<float> *d_f = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto cleanup = [&]() {
        void *ptrs[] = {G.bmap, d_a, d_t, d_f};
        for (void *q : ptrs) if (q) cudaFree(q);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    };
    struct Guard { std::function<void()> f; ~Guard() { f(); } } guard{cleanup};
    if ((rc = dev_upload(&G.bmap, m)) || (rc = dev_upload(&d_a, a)) || (rc = dev_upload(&d_t, t)) ||
        (rc = dev_upload(&d_f, f)))
        return rc;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const dim3 fgrid(64, k);
    auto once = [&]() -> int {
        int r2 = launch_batched<float>(bs, G, d_a, d_t, 1, 0);
        if (r2) return r2;
        fixup_batched_kernel<float><<<fgrid, 128, 0, bs>>>(d_f, 1, 0);
        CK(cudaGetLastError());
        return FG_OK;
    };
    for (int w = 0; w < 2; ++w)
        if ((rc = once())) return rc;
    CK(cudaEventRecord(e0, bs));
    for (int r = 0; r < reps; ++r)
        if ((rc = once())) return rc;
    CK(cudaEventRecord(e1, bs));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    *us = 1e3 * ms / reps;
    for (int j = 0; j < k; ++j)
        if ((rc = check_device_error(ops[inst[j]]))) return rc;
    return FG_OK;
}

extern "C" {

FG_API int fg_op_set_tile(fg_op *op, int tz) {
    FG_NEED_BOX(op, "fg_op_set_tile");
    if (!op) return fail(FG_INVALID_ARGUMENT, "NULL op");
    if (tz < 1 || tz > 64) return fail(FG_INVALID_ARGUMENT, "tile depth %d outside 1..64", tz);
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    return set_tile_locked(op, tz);
}

FG_API int fg_op_tile(const fg_op *op, int dims[3]) {
    FG_NEED_BOX(op, "fg_op_tile");
    if (!op || !dims) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    dims[0] = 32;
    dims[1] = op->g.WY;
    dims[2] = op->g.TZ;
    return FG_OK;
}

FG_API int fg_batch_autotune(fg_op *const *ops, int n, int reps, fg_tune_entry *out, int max_out, int *n_out) {
    if (ops)
        for (int i_ = 0; i_ < n; ++i_) FG_NEED_BOX(ops[i_], "fg_batch_autotune");
    if (!ops || n <= 0 || reps < 1 || !n_out) return fail(FG_INVALID_ARGUMENT, "bad autotune arguments");
    *n_out = 0;
    std::vector<fg_op *> sorted(ops, ops + n);
    for (int i = 0; i < n; ++i)
        if (!ops[i]) return fail(FG_INVALID_ARGUMENT, "NULL instance %d", i);
    std::sort(sorted.begin(), sorted.end());
    if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
        return fail(FG_INVALID_ARGUMENT, "an operator appears twice in the batch");
    std::vector<std::unique_lock<std::mutex>> locks;
    for (fg_op *o : sorted) locks.emplace_back(o->mu);
    const int dev = ops[0]->device;
    for (int i = 0; i < n; ++i)
        if (ops[i]->device != dev) return fail(FG_INVALID_ARGUMENT, "batch spans devices");
    CK(cudaSetDevice(dev));
    int rc;
    for (int i = 0; i < n; ++i)
        if ((rc = ensure_solver_buffers(ops[i])) || (rc = ensure_fp32(ops[i]))) return rc;
    // classes of (order, kind, size): elements <= 16^3, <= 32^3, larger; the
    // quadrature-data format is a tuned dimension of each class
    struct Cls { int p, kind, sc; std::vector<int> inst; };
    std::vector<Cls> cls;
    for (int i = 0; i < n; ++i) {
        const fg_op *o = ops[i];
        const int64_t E = (int64_t)o->g.nx * o->g.ny * o->g.nz;
        const int sc = E <= 4096 ? 0 : (E <= 32768 ? 1 : 2);
        auto it = std::find_if(cls.begin(), cls.end(), [&](const Cls &c) {
            return c.p == o->p && c.kind == o->kind && c.sc == sc;
        });
        if (it == cls.end()) { cls.push_back(Cls{o->p, o->kind, sc, {}}); it = cls.end() - 1; }
        it->inst.push_back(i);
    }
    cudaStream_t bs;
    CK(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking));
    struct SG { cudaStream_t s; ~SG() { cudaStreamDestroy(s); } } sg{bs};
    // depth of a candidate for one instance: at most the largest power of two <= nz
    auto depth = [&](const fg_op *o, int tz) {
        int d = 1;
        while (d * 2 <= tz && d * 2 <= o->g.nz) d *= 2;
        return d;
    };
    // put every member of a class on format f; false if a member refuses the
    // affine format (an element whose Jacobian is not constant)
    auto set_format = [&](const Cls &c, int f, int &err) {
        err = FG_OK;
        for (int i : c.inst) {
            fg_op *o = ops[i];
            if (f == 1 && !o->qa64) {
                const int r = build_affine<double>(o, &o->qa64);
                if (r == FG_UNSUPPORTED) {
                    t_last_status = FG_OK;  // a refusal here only removes the candidate
                    for (int j : c.inst) ops[j]->fmt = 0;
                    return false;
                }
                if (r) { err = r; return false; }
            }
            o->fmt = f;
        }
        return true;
    };
    int count = 0;
    for (const Cls &c : cls) {
        double us[2][FG_TUNE_CANDIDATES];
        int best_f = -1, best_k = -1;
        int maxnz = 1;
        for (int i : c.inst) maxnz = std::max(maxnz, ops[i]->g.nz);
        for (int f = 0; f < 2; ++f) {
            for (int k = 0; k < FG_TUNE_CANDIDATES; ++k) us[f][k] = -1.0;
            int err;
            if (!set_format(c, f, err)) {
                if (err) return err;
                continue;
            }
            for (int k = 0; k < FG_TUNE_CANDIDATES; ++k) {
                if (k > 0 && kTuneTZ[k] > maxnz) continue;  // same shapes as a smaller candidate
                for (int i : c.inst)
                    if ((rc = set_tile_locked(ops[i], depth(ops[i], kTuneTZ[k])))) return rc;
                if ((rc = time_batched_apply(ops, c.inst, bs, reps, &us[f][k]))) return rc;
                if (best_k < 0 || us[f][k] < us[best_f][best_k]) {
                    best_f = f;
                    best_k = k;
                }
            }
        }
        int err;
        if (!set_format(c, best_f, err)) return err ? err : fail(FG_CUDA_ERROR, "autotune: format lost");
        for (int i : c.inst) {
            if ((rc = set_tile_locked(ops[i], depth(ops[i], kTuneTZ[best_k]))) || (rc = ensure_fp32(ops[i])))
                return rc;
            CK(cudaStreamSynchronize(ops[i]->stream));
        }
        if (out && count < max_out) {
            fg_tune_entry &e = out[count];
            e.order = c.p;
            e.kind = c.kind;
            e.size_class = c.sc;
            e.instances = (int)c.inst.size();
            e.tz = kTuneTZ[best_k];
            e.format = best_f;
            for (int k = 0; k < FG_TUNE_CANDIDATES; ++k) {
                e.us[k] = us[best_f][k];
                e.us_other[k] = us[1 - best_f][k];
            }
        }
        ++count;
    }
    *n_out = count;
    return FG_OK;
}

}  // extern "C"

extern "C" {

FG_API int fg_pcg(fg_op *op, const double *b, double *x, const fg_cfg *cfg_in, fg_result *res,
                  int mem) {
    if (!op || !b || !x) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    fg_cfg cfg;
    if (cfg_in) cfg = *cfg_in; else fg_cfg_default(&cfg);
    int rc;
    if ((rc = validate_cfg(cfg))) return rc;
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    if ((rc = ensure_solver_buffers(op))) return rc;
    if ((rc = to_native(op, op->bw, b, mem)) || (rc = to_native(op, op->xw, x, mem))) return rc;
    const int status = pcg_core(op, cfg, res);
    if (status != FG_OK && status != FG_CONVERGENCE_FAILED && status != FG_BREAKDOWN) return status;
    if ((rc = from_native(op, x, op->xw, mem))) return rc;
    CK(cudaStreamSynchronize(op->stream));
    if (status != FG_OK) {  // restore the solver's message
        if (status == FG_BREAKDOWN) fail(status, "CG breakdown: p^T A p is near zero");
        else fail(status, "solver did not converge in %d iterations", cfg.max_iter);
    }
    return status;
}

// Batched solves (hundreds of uneven instances): every operator is solved by the
// mixed-precision PCG (FP32 applies and smoother, FP64 reliable updates and
// dot products) of fg_pcg, but each phase of an iteration is one launch over
// all instances (per order/kind/format group for the applies), converged
// instances are masked per instance on the device, and chunks of
// check_interval iterations are captured once in a CUDA graph and replayed.
FG_API int fg_batch_pcg(fg_op *const *ops, int n, const double *const *b, double *const *x,
                        const fg_cfg *cfg_in, fg_result *results, int mem) {
    if (ops)
        for (int i_ = 0; i_ < n; ++i_) FG_NEED_BOX(ops[i_], "fg_batch_pcg");
    if (!ops || n <= 0 || !b || !x) return fail(FG_INVALID_ARGUMENT, "bad batch arguments");
    fg_cfg cfg;
    if (cfg_in) cfg = *cfg_in; else fg_cfg_default(&cfg);
    int rc;
    if ((rc = validate_cfg(cfg))) return rc;
    if (cfg.precision != FG_FP32_IR)
        return fail(FG_UNSUPPORTED, "batched solves run the FP32 mixed-precision form only");
    if (cfg.precond != FG_PC_JACOBI && cfg.precond != FG_PC_CHEBYSHEV)
        return fail(FG_UNSUPPORTED, "batched solves need the Jacobi or Chebyshev preconditioner");
    const bool cheb = cfg.precond == FG_PC_CHEBYSHEV;
    if (cheb && cfg.cheb_degree > BATCH_MAXK) return fail(FG_INVALID_ARGUMENT, "cheb_degree too large");
    std::vector<fg_op *> sorted(ops, ops + n);
    for (int i = 0; i < n; ++i)
        if (!ops[i] || !b[i] || !x[i]) return fail(FG_INVALID_ARGUMENT, "NULL instance %d", i);
    std::sort(sorted.begin(), sorted.end());
    if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
        return fail(FG_INVALID_ARGUMENT, "an operator appears twice in the batch");
    std::vector<std::unique_lock<std::mutex>> locks;
    for (fg_op *o : sorted) locks.emplace_back(o->mu);
    const int dev = ops[0]->device;
    for (int i = 0; i < n; ++i)
        if (ops[i]->device != dev) return fail(FG_INVALID_ARGUMENT, "batch spans devices");
    CK(cudaSetDevice(dev));
    // per-instance preparation on each operator's own stream
    std::vector<double> lmax(n, 0.0);
    for (int i = 0; i < n; ++i) {
        fg_op *o = ops[i];
        if ((rc = ensure_solver_buffers(o)) || (rc = ensure_fp32(o)) || (rc = ensure_dinv32(o))) return rc;
        if (cheb) {
            if (cfg.lmax > 0) lmax[i] = cfg.lmax;
            else {
                if (!o->have_lmax) {
                    if ((rc = estimate_lmax(o, cfg.power_iters > 0 ? cfg.power_iters : 20, &o->lmax_est)))
                        return rc;
                    o->have_lmax = true;
                }
                lmax[i] = (cfg.lmax_safety > 0 ? cfg.lmax_safety : 1.1) * o->lmax_est;
            }
        }
        if ((rc = to_native(o, o->bw, b[i], mem)) || (rc = to_native(o, o->xw, x[i], mem))) return rc;
        CK(cudaStreamSynchronize(o->stream));
    }
    cudaStream_t bs;
    CK(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking));
    // device tables
    constexpr int VBX = 64;
    std::vector<ApplyArgs<float>> a32(2 * n);
    std::vector<ApplyArgs<double>> a64(n);
    std::vector<CUtensorMap> t32(2 * n), t64(n);
    std::vector<FixArgs<float>> f32(2 * n);
    std::vector<FixArgs<double>> f64(n);
    std::vector<BatchVec> bv(n);
    SolverState *d_st = nullptr;
    double *d_part = nullptr;
    CK(cudaMalloc(&d_st, sizeof(SolverState) * n));
    CK(cudaMalloc(&d_part, sizeof(double) * 2 * VBX * n));
    std::vector<SolverState> hst(n);
    for (int i = 0; i < n; ++i) {
        fg_op *o = ops[i];
        Grid g = o->g;
        g.ess = o->ess_tags;
        const float *q32 = qdata_of<float>(o);
        const double *q64 = qdata_of<double>(o);
        a32[2 * i] = ApplyArgs<float>{g, q32, o->ap32, o->face32, 0, o->d_err, &d_st[i].done};
        a32[2 * i + 1] = ApplyArgs<float>{g, q32, o->ct32, o->face32, 0, o->d_err, &d_st[i].done};
        a64[i] = ApplyArgs<double>{g, q64, o->ap, o->face, 0, o->d_err, &d_st[i].skip_rel};
        if ((rc = encode_xmap<float>(o, o->p32, &t32[2 * i])) ||
            (rc = encode_xmap<float>(o, o->cd32, &t32[2 * i + 1])) ||
            (rc = encode_xmap<double>(o, o->xw, &t64[i])))
            return rc;
        f32[2 * i] = FixArgs<float>{g, o->ap32, o->face32, &d_st[i].done};
        f32[2 * i + 1] = FixArgs<float>{g, o->ct32, o->face32, &d_st[i].done};
        f64[i] = FixArgs<double>{g, o->ap, o->face, &d_st[i].skip_rel};
        BatchVec &B = bv[i];
        B.n = o->Nn;
        B.x64 = o->xw; B.b64 = o->bw; B.ap64 = o->ap;
        B.r = o->r32; B.z = o->z32; B.p = o->p32; B.ap = o->ap32; B.e = o->e32;
        B.cres = o->cres32; B.cd = o->cd32; B.ct = o->ct32; B.dinv = o->dinv32;
        B.partials = d_part + (size_t)2 * VBX * i;
        B.st = &d_st[i];
        if (cheb) {
            const ChebCoef cc = cheb_coefs(lmax[i] / (cfg.lmin_ratio > 0 ? cfg.lmin_ratio : 30.0), lmax[i],
                                           cfg.cheb_degree);
            B.inv_theta = cc.inv_theta;
            for (size_t k = 0; k < cc.c1.size(); ++k) { B.c1[k] = cc.c1[k]; B.c2[k] = cc.c2[k]; }
        }
        SolverState &h = hst[i];
        h = SolverState{};
        h.rtol = cfg.rtol; h.atol = cfg.atol; h.max_iter = cfg.max_iter;
        h.delta = (cfg.inner_rtol > 0 && cfg.inner_rtol < 1) ? cfg.inner_rtol : 0.1;
        h.skip_rel = 0;  // the initial FP64 residual always runs
    }
    // groups of equal (order, kind, format); block maps
    std::vector<BatchGroup> groups;
    for (int i = 0; i < n; ++i) {
        fg_op *o = ops[i];
        auto it = std::find_if(groups.begin(), groups.end(), [&](const BatchGroup &G) {
            return G.p == o->p && G.kind == o->kind && G.fmt == o->fmt;
        });
        if (it == groups.end()) { groups.push_back(BatchGroup{o->p, o->kind, o->fmt, {}}); it = groups.end() - 1; }
        it->inst.push_back(i);
    }
    ApplyArgs<float> *d_a32 = nullptr;
    ApplyArgs<double> *d_a64 = nullptr;
    CUtensorMap *d_t32 = nullptr, *d_t64 = nullptr;
    FixArgs<float> *d_f32 = nullptr;
    FixArgs<double> *d_f64 = nullptr;
    BatchVec *d_bv = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    auto cleanup = [&]() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        for (auto &G : groups) if (G.bmap) cudaFree(G.bmap);
        void *ptrs[] = {d_a32, d_a64, d_t32, d_t64, d_f32, d_f64, d_bv, d_st, d_part};
        for (void *p : ptrs) if (p) cudaFree(p);
        cudaStreamDestroy(bs);
    };
    struct Guard { std::function<void()> f; ~Guard() { f(); } } guard{cleanup};
    for (auto &G : groups) {
        const std::vector<int2> m = largest_first_bmap(ops, G.inst, G.inst);
        G.nblocks = (int)m.size();
        if ((rc = dev_upload(&G.bmap, m))) return rc;
    }
    if ((rc = dev_upload(&d_a32, a32)) || (rc = dev_upload(&d_a64, a64)) || (rc = dev_upload(&d_t32, t32)) ||
        (rc = dev_upload(&d_t64, t64)) || (rc = dev_upload(&d_f32, f32)) || (rc = dev_upload(&d_f64, f64)) ||
        (rc = dev_upload(&d_bv, bv)))
        return rc;
    CK(cudaMemcpy(d_st, hst.data(), sizeof(SolverState) * n, cudaMemcpyHostToDevice));
    FG_LEGACY_FENCE();
    const dim3 vgrid(VBX, n), fgrid(64, n);
    auto apply32 = [&](int slot) -> int {
        for (auto &G : groups) {
            int r2 = launch_batched<float>(bs, G, d_a32, d_t32, 2, slot);
            if (r2) return r2;
        }
        fixup_batched_kernel<float><<<fgrid, 128, 0, bs>>>(d_f32, 2, slot);
        CK(cudaGetLastError());
        return FG_OK;
    };
    auto apply64 = [&]() -> int {
        for (auto &G : groups) {
            int r2 = launch_batched<double>(bs, G, d_a64, d_t64, 1, 0);
            if (r2) return r2;
        }
        fixup_batched_kernel<double><<<fgrid, 128, 0, bs>>>(d_f64, 1, 0);
        CK(cudaGetLastError());
        return FG_OK;
    };
    auto precond = [&](int init) -> int {
        if (cheb) {
            kb_cheb_first<<<vgrid, VEC_THREADS, 0, bs>>>(d_bv);
            for (int sidx = 0; sidx + 1 < cfg.cheb_degree; ++sidx) {
                int r2 = apply32(1);
                if (r2) return r2;
                kb_cheb_step<<<vgrid, VEC_THREADS, 0, bs>>>(d_bv, sidx, sidx + 2 == cfg.cheb_degree ? 1 : 0);
            }
            kb_rz<<<vgrid, VEC_THREADS, 0, bs>>>(d_bv, init, 0);
        } else {
            kb_rz<<<vgrid, VEC_THREADS, 0, bs>>>(d_bv, init, 1);
        }
        kb_pupdate<<<vgrid, VEC_THREADS, 0, bs>>>(d_bv, init);
        CK(cudaGetLastError());
        return FG_OK;
    };
    for (auto &G : groups)  // kernel attributes are set outside the graph capture
        if ((rc = launch_batched<float>(bs, G, nullptr, nullptr, 2, 0)) ||
            (rc = launch_batched<double>(bs, G, nullptr, nullptr, 1, 0)))
            return rc;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    CK(cudaEventRecord(e0, bs));
    kb_zero_e<<<vgrid, VEC_THREADS, 0, bs>>>(d_bv);
    if ((rc = apply64())) return rc;
    kb_rel_residual<<<vgrid, VEC_THREADS, 0, bs>>>(d_bv, 1);
    if ((rc = precond(1))) return rc;
    // one chunk of iterations, captured once and replayed
    const int chunk = std::max(1, cfg.check_interval);
    CK(cudaStreamBeginCapture(bs, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < chunk; ++k) {
        if ((rc = apply32(0))) { cudaStreamEndCapture(bs, &graph); return rc; }
        kb_pap<<<vgrid, VEC_THREADS, 0, bs>>>(d_bv);
        kb_rel_step<<<vgrid, VEC_THREADS, 0, bs>>>(d_bv);
        kb_rel_xupdate<<<vgrid, VEC_THREADS, 0, bs>>>(d_bv);
        if ((rc = apply64())) { cudaStreamEndCapture(bs, &graph); return rc; }
        kb_rel_residual<<<vgrid, VEC_THREADS, 0, bs>>>(d_bv, 0);
        if ((rc = precond(0))) { cudaStreamEndCapture(bs, &graph); return rc; }
    }
    CK(cudaStreamEndCapture(bs, &graph));
    CK(cudaGraphInstantiate(&gexec, graph, 0));
    int launched = 0;
    while (launched < cfg.max_iter) {
        CK(cudaGraphLaunch(gexec, bs));
        launched += chunk;
        CK(cudaMemcpyAsync(hst.data(), d_st, sizeof(SolverState) * n, cudaMemcpyDeviceToHost, bs));
        CK(cudaStreamSynchronize(bs));
        bool all = true;
        for (int i = 0; i < n && all; ++i) all = hst[i].done != 0;
        if (all) break;
    }
    CK(cudaEventRecord(e1, bs));
    // true residuals in FP64 (every instance)
    for (int i = 0; i < n; ++i) hst[i].skip_rel = 0;
    for (int i = 0; i < n; ++i)
        CK(cudaMemcpyAsync(&d_st[i].skip_rel, &hst[i].skip_rel, sizeof(int), cudaMemcpyHostToDevice, bs));
    if ((rc = apply64())) return rc;
    kb_true_residual<<<vgrid, VEC_THREADS, 0, bs>>>(d_bv);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(hst.data(), d_st, sizeof(SolverState) * n, cudaMemcpyDeviceToHost, bs));
    CK(cudaStreamSynchronize(bs));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int nfail = 0;
    for (int i = 0; i < n; ++i) {
        fg_op *o = ops[i];
        if ((rc = from_native(o, x[i], o->xw, mem))) return rc;
        const SolverState &h = hst[i];
        const int status = h.converged ? FG_OK : (h.breakdown ? FG_BREAKDOWN : FG_CONVERGENCE_FAILED);
        if (status != FG_OK) ++nfail;
        if (results) {
            fg_result &r = results[i];
            r.converged = h.converged;
            r.iterations = h.converged ? h.iter : (h.breakdown ? h.iter : cfg.max_iter);
            r.final_residual = h.res;
            r.true_residual = h.tmp[0];
            r.status = status;
            r.outer_iterations = (int)h.tmp[1];
            r.applies = (int64_t)h.iter * (1 + (cheb ? cfg.cheb_degree - 1 : 0));
            r.lmax = lmax[i];
            r.solve_ms = ms;
        }
    }
    for (int i = 0; i < n; ++i) CK(cudaStreamSynchronize(ops[i]->stream));
    for (int i = 0; i < n; ++i)
        if ((rc = check_device_error(ops[i]))) return rc;
    if (nfail) return fail(FG_CONVERGENCE_FAILED, "%d of %d batched solves did not converge", nfail, n);
    t_last_status = FG_OK;
    return FG_OK;
}

// SDIRK-2 heat stepping (examples/mfem_ex10_heat_equation.rs:201-250,
// gamma = 1 - 1/sqrt(2) as crates/solver/src/ode.rs:441): M u_t + K u = 0,
// homogeneous Dirichlet.  Per step:
//   (M + g dt K) k1 = -K u,          u2 = u + dt (1-g) k1,
//   (M + g dt K) k2 = -K u2,         u += dt ((1-g) k1 + g k2).
// Stage solves run on the device with the PCG core, warm-started from the
// previous stage's k (the reference starts every solve from zero).
FG_API int fg_sdirk2(fg_op *stiff, fg_op *stage, double *u, double dt, int n_steps,
                     const fg_cfg *cfg_in, fg_sdirk_result *out, int mem) {
    FG_NEED_BOX(stiff, "fg_sdirk2");
    FG_NEED_BOX(stage, "fg_sdirk2");
    if (!stiff || !stage || !u) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (stiff == stage) return fail(FG_INVALID_ARGUMENT, "stiff and stage must be distinct handles");
    if (n_steps < 0 || !(dt > 0)) return fail(FG_INVALID_ARGUMENT, "bad dt or n_steps");
    if (stiff->device != stage->device || stiff->N != stage->N || stiff->g.NI != stage->g.NI ||
        stiff->g.NJ != stage->g.NJ || stiff->g.NK != stage->g.NK || stiff->p != stage->p)
        return fail(FG_DIMENSION_MISMATCH, "stiff and stage operators live on different meshes");
    fg_cfg cfg;
    if (cfg_in) cfg = *cfg_in; else fg_cfg_default(&cfg);
    int rc;
    if ((rc = validate_cfg(cfg))) return rc;
    std::scoped_lock lk(stiff->mu, stage->mu);
    CK(cudaSetDevice(stage->device));
    cudaStream_t saved = stiff->stream;
    stiff->stream = stage->stream;  // one stream orders both operators' work
    struct Restore { fg_op *o; cudaStream_t s; ~Restore() { o->stream = s; } } restore{stiff, saved};
    CK(cudaStreamSynchronize(saved));
    if ((rc = ensure_solver_buffers(stage))) return rc;
    for (double **b : {&stage->sd_u, &stage->sd_k1, &stage->sd_w})
        if (!*b && (rc = alloc_vec(b, stage->Nn))) return rc;
    const int64_t n = stage->Nn;
    const double g = 1.0 - std::sqrt(0.5);
    if ((rc = to_native(stage, stage->sd_u, u, mem))) return rc;
    CK(cudaMemsetAsync(stage->xw, 0, sizeof(double) * n, stage->stream));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    CK(cudaEventRecord(e0, stage->stream));
    int64_t total_it = 0, applies = 0;
    int max_it = 0, failed = 0;
    // Each stage is solved for b/||b|| (and the warm start scaled alike), then
    // scaled back: CG is scale-invariant, but the reference's absolute
    // breakdown test |p^T A p| < 1e-30 (par_solver.rs:294) would otherwise trip
    // once the decaying solution makes the stage right-hand sides tiny.
    double *scal = nullptr;  // ||b|| kept in a device scalar between the two calls
    auto normalise = [&](bool before) -> int {
        if (before) {
            k_norm_tmp<<<VEC_GRID, VEC_THREADS, 0, stage->stream>>>(n, stage->bw, stage->partials, stage->st);
            k_scale_tmp<<<VEC_GRID, VEC_THREADS, 0, stage->stream>>>(n, stage->bw, stage->st, 1);
            k_scale_tmp<<<VEC_GRID, VEC_THREADS, 0, stage->stream>>>(n, stage->xw, stage->st, 1);
            CK(cudaMemcpyAsync(scal, &stage->st->tmp[2], sizeof(double), cudaMemcpyDeviceToDevice,
                               stage->stream));
        } else {
            CK(cudaMemcpyAsync(&stage->st->tmp[2], scal, sizeof(double), cudaMemcpyDeviceToDevice,
                               stage->stream));
            k_scale_tmp<<<VEC_GRID, VEC_THREADS, 0, stage->stream>>>(n, stage->xw, stage->st, 0);
        }
        CK(cudaGetLastError());
        return FG_OK;
    };
    CK(cudaMalloc(&scal, sizeof(double)));
    struct FreeScal { double *p; ~FreeScal() { cudaFree(p); } } free_scal{scal};
    auto stage_solve = [&](const double *ucur) -> int {
        int r2 = apply_native(stiff, ucur, stage->sd_w, 0, 1, nullptr);
        if (r2) return r2;
        ++applies;
        k_lincomb2<<<VEC_GRID, VEC_THREADS, 0, stage->stream>>>(n, stage->bw, -1.0, stage->sd_w, 0.0,
                                                                 stage->sd_w);
        CK(cudaGetLastError());
        fg_result r{};
        int st = normalise(true);
        if (st) return st;
        st = pcg_core(stage, cfg, &r);
        if (st != FG_OK && st != FG_CONVERGENCE_FAILED && st != FG_BREAKDOWN) return st;
        if (int s2 = normalise(false)) return s2;
        if (st != FG_OK) ++failed;
        total_it += r.iterations;
        applies += r.applies;
        max_it = std::max(max_it, (int)r.iterations);
        return FG_OK;
    };
    for (int step = 0; step < n_steps; ++step) {
        if ((rc = stage_solve(stage->sd_u))) return rc;                 // k1 in xw
        CK(cudaMemcpyAsync(stage->sd_k1, stage->xw, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                           stage->stream));
        // u2 = u + dt (1-g) k1 (held in the solver's r buffer until the stiff apply reads it)
        k_lincomb2<<<VEC_GRID, VEC_THREADS, 0, stage->stream>>>(n, stage->r, 1.0, stage->sd_u,
                                                                 dt * (1.0 - g), stage->sd_k1);
        if ((rc = apply_native(stiff, stage->r, stage->sd_w, 0, 1, nullptr))) return rc;
        ++applies;
        k_lincomb2<<<VEC_GRID, VEC_THREADS, 0, stage->stream>>>(n, stage->bw, -1.0, stage->sd_w, 0.0,
                                                                 stage->sd_w);
        {
            fg_result r{};
            int st = normalise(true);
            if (st) return st;
            st = pcg_core(stage, cfg, &r);                               // k2 in xw (warm: k1)
            if (st != FG_OK && st != FG_CONVERGENCE_FAILED && st != FG_BREAKDOWN) return st;
            if (int s2 = normalise(false)) return s2;
            if (st != FG_OK) ++failed;
            total_it += r.iterations;
            applies += r.applies;
            max_it = std::max(max_it, (int)r.iterations);
        }
        // u += dt (1-g) k1 + dt g k2
        k_lincomb2<<<VEC_GRID, VEC_THREADS, 0, stage->stream>>>(n, stage->sd_w, dt * (1.0 - g),
                                                                 stage->sd_k1, dt * g, stage->xw);
        k_lincomb2<<<VEC_GRID, VEC_THREADS, 0, stage->stream>>>(n, stage->sd_u, 1.0, stage->sd_u, 1.0,
                                                                 stage->sd_w);
        CK(cudaGetLastError());
    }
    CK(cudaEventRecord(e1, stage->stream));
    if ((rc = from_native(stage, u, stage->sd_u, mem))) return rc;
    CK(cudaStreamSynchronize(stage->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (out) {
        out->steps = n_steps;
        out->total_iterations = total_it;
        out->max_stage_iterations = max_it;
        out->failed_solves = failed;
        out->applies = applies;
        out->time_ms = ms;
    }
    if ((rc = check_device_error(stage))) return rc;
    if (failed) return fail(FG_CONVERGENCE_FAILED, "%d stage solves did not converge", failed);
    t_last_status = FG_OK;
    return FG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Solver steps on caller-owned device vectors of a handle's native layout, for
// loops whose dot products are completed outside the library (the sharded
// PCG of crates/parallel/src/par_solver.rs:262-342: each rank's owned-DOF dots,
// then the caller's allreduce, ParVector::global_dot, par_vector.rs:182-194).
// The scalars stay in device memory; everything runs on the handle's stream.
// ---------------------------------------------------------------------------
extern "C" {

FG_API int fg_vec_dots(fg_op *op, int64_t n_own, int npairs, const double *const *a, const double *const *b,
                       double *out) {
    if (!op || !a || !b || !out) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (npairs < 1 || npairs > 3) return fail(FG_INVALID_ARGUMENT, "1 to 3 pairs");
    if (n_own < 0 || n_own > op->Nn || n_own % 4) return fail(FG_INVALID_ARGUMENT, "n_own must be a multiple "
                                                             "of 4 within the native length");
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    VecPairs P{};
    for (int j = 0; j < npairs; ++j) {
        if (!a[j] || !b[j]) return fail(FG_INVALID_ARGUMENT, "NULL vector");
        P.a[j] = a[j];
        P.b[j] = b[j];
    }
    switch (npairs) {
    case 1: k_sh_dots<1><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n_own, P, op->partials, op->st, out); break;
    case 2: k_sh_dots<2><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n_own, P, op->partials, op->st, out); break;
    default: k_sh_dots<3><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n_own, P, op->partials, op->st, out); break;
    }
    CK(cudaGetLastError());
    return FG_OK;
}

FG_API int fg_vec_pcg_update(fg_op *op, int64_t n_own, double *x, double *r, const double *p, const double *ap,
                             const double *dinv, double *z, const double *rz_pap, double *rr_rz) {
    if (!op || !x || !r || !p || !ap || !dinv || !z || !rz_pap || !rr_rz)
        return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (n_own < 0 || n_own > op->Nn || n_own % 4) return fail(FG_INVALID_ARGUMENT, "n_own must be a multiple "
                                                             "of 4 within the native length");
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    k_sh_update<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(op->Nn, n_own, x, r, p, ap, dinv, z, rz_pap,
                                                          op->partials, op->st, rr_rz);
    CK(cudaGetLastError());
    return FG_OK;
}

FG_API int fg_vec_pupdate(fg_op *op, const double *z, double *p, const double *num, const double *den) {
    if (!op || !z || !p || !num || !den) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    k_sh_pupdate<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(op->Nn, z, p, num, den);
    CK(cudaGetLastError());
    return FG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free apply.
//
// Same kernels as fg_op_apply_native, but the face-slot scratch that the
// fix-up pass reads comes from a fixed array compiled into this library
// instead of the handle's own buffer, so the call neither allocates nor
// depends on allocator state.  The array lives in every GPU context that
// loads the library until the process exits.
// ---------------------------------------------------------------------------
#define FG_NOALLOC_FACE_DOUBLES (4u << 20)  // 4 Mi doubles = 32 MiB
static __device__ __align__(256) double g_noalloc_face[FG_NOALLOC_FACE_DOUBLES];
// device address of g_noalloc_face per device, with the context it was resolved in
static double *g_noalloc_face_ptr[64];
static CUcontext g_noalloc_ctx[64];
static std::mutex g_noalloc_mu;
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
static CtxGetCurrentFn g_ctx_get_current = nullptr;

// Host code cannot use g_noalloc_face directly (its host-side name is only a
// stand-in for the symbol); resolve the device address with that device
// current.  The address belongs to the context the module was loaded in: it
// is resolved again when the current context differs from the one it was
// resolved in (after cudaDeviceReset, or when the primary context was released
// and created anew), so a stale address is never passed to a kernel.
static int noalloc_scratch(int dev, double **out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (dev < 0 || dev >= 64) return fail(FG_CUDA_ERROR, "device id %d out of range", dev);
    if (!g_ctx_get_current) {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        CK(cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn)
            return fail(FG_CUDA_ERROR, "cuCtxGetCurrent entry point not found");
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
    }
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx)
        return fail(FG_CUDA_ERROR, "no current CUDA context on device %d", dev);
    if (!g_noalloc_face_ptr[dev] || g_noalloc_ctx[dev] != ctx) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_face);
        if (e != cudaSuccess || !p)
            return fail(FG_CUDA_ERROR, "cudaGetSymbolAddress(g_noalloc_face) failed: %s",
                        cudaGetErrorString(e));
        g_noalloc_face_ptr[dev] = static_cast<double *>(p);
        g_noalloc_ctx[dev] = ctx;
    }
    *out = g_noalloc_face_ptr[dev];
    return FG_OK;
}

template <int P, int OPK>
static int noalloc_launch_apply_t(fg_op *op, const Grid &g, const double *x, double *y,
                                  int accumulate, double *face) {
    using C = KCfg<P>;
    using SM = ApplySmem<P, double, C::WY, C::S, stage_elems<P, OPK, 0>() / 32>;
    auto kern = pa_apply_kernel<P, OPK, double, C::WY, C::S, C::MINB>;
    // per device, set once (as launch_apply_t does); racing setters are harmless
    static std::atomic<bool> attr_set[64];
    if (op->device < 0 || op->device >= 64) return fail(FG_CUDA_ERROR, "device id %d out of range", op->device);
    if (!attr_set[op->device].load(std::memory_order_acquire)) {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SM::bytes));
        attr_set[op->device].store(true, std::memory_order_release);
    }
    CUtensorMap tmap;
    cuuint64_t gdim[3] = {(cuuint64_t)g.NI, (cuuint64_t)g.NJ, (cuuint64_t)g.NK};
    cuuint64_t gstr[2] = {(cuuint64_t)g.NIp * sizeof(double),
                          (cuuint64_t)g.NIp * g.NJ * sizeof(double)};
    cuuint32_t box[3] = {(cuuint32_t)SM::XW, (cuuint32_t)SM::RY, (cuuint32_t)(P + 1)};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult cr = g_encode(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(x), gdim,
                           gstr, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return fail(FG_CUDA_ERROR, "cuTensorMapEncodeTiled failed (%d)", (int)cr);
    ApplyArgs<double> A{g, op->qd, y, face, accumulate, op->d_err, nullptr, nullptr, op->wait_ns};
    kern<<<g.n_items(), C::WY * 32, SM::bytes, op->stream>>>(tmap, A);
    CK(cudaGetLastError());
    return FG_OK;
}

template <int P>
static int noalloc_launch_apply_p(fg_op *op, const Grid &g, const double *x, double *y,
                                  int accumulate, double *face) {
    switch (op->kind) {
    case FG_MASS: return noalloc_launch_apply_t<P, 1>(op, g, x, y, accumulate, face);
    case FG_DIFF: return noalloc_launch_apply_t<P, 2>(op, g, x, y, accumulate, face);
    default: return noalloc_launch_apply_t<P, 3>(op, g, x, y, accumulate, face);
    }
}

extern "C" FG_API int fg_op_apply_native_noalloc(fg_op *op, const double *x, double *y,
                                                 int accumulate, int constrained) {
    FG_NEED_BOX(op, "fg_op_apply_native_noalloc");
    if (!op || !x || !y) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (x == y) return fail(FG_INVALID_ARGUMENT, "x and y must not alias");
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    Grid g = op->g;
    g.ess = constrained ? op->ess_tags : 0;
    const size_t need = (size_t)g.n_items() * (size_t)g.face_stride();
    if (need > FG_NOALLOC_FACE_DOUBLES)
        return fail(FG_INVALID_ARGUMENT,
                    "fg_op_apply_native_noalloc: this operator needs %zu doubles of face scratch, "
                    "more than the %u (32 MiB) of the static scratch array; use fg_op_apply_native",
                    need, (unsigned)FG_NOALLOC_FACE_DOUBLES);
    double *face = nullptr;
    int rc = noalloc_scratch(op->device, &face);
    if (rc) return rc;
    // Every face slot the fix-up reads is written by the apply kernel earlier in
    // the same call, so stale contents from a previous call need no clearing.
    switch (op->p) {
    case 1: rc = noalloc_launch_apply_p<1>(op, g, x, y, accumulate, face); break;
    case 2: rc = noalloc_launch_apply_p<2>(op, g, x, y, accumulate, face); break;
    default: rc = noalloc_launch_apply_p<3>(op, g, x, y, accumulate, face); break;
    }
    if (rc) return rc;
    const dim3 grid = fixup_grid(g);
    if (grid.x > 0) {
        fixup_kernel<double><<<grid, 128, 0, op->stream>>>(g, y, face, nullptr);
        CK(cudaGetLastError());
    }
    return FG_OK;
}

// ---------------------------------------------------------------------------
// Learned coarse correction: network handle, training, attachment.
// ---------------------------------------------------------------------------
static int unet_params_layout(const fg_unet *u, std::vector<int64_t> *offs) {
    int64_t o = 0;
    for (int l = 0; l < NLAYERS; ++l) {
        offs->push_back(o);
        o += (int64_t)u->L[l].cout * 27 * u->L[l].cin + u->L[l].cout;
    }
    offs->push_back(o);
    return FG_OK;
}

static int unet_copy_params(fg_unet *u, float *host, bool to_host, bool grads) {
    for (int l = 0; l < NLAYERS; ++l) {
        ConvLayer &L = u->L[l];
        const int K = 27 * L.cin;
        float *w = grads ? L.gw : L.w, *b = grads ? L.gb : L.b;
        if (to_host) {
            CK(cudaMemcpy2D(host, K * sizeof(float), w, L.kp * sizeof(float), K * sizeof(float), L.cout,
                            cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(host + (int64_t)L.cout * K, b, L.cout * sizeof(float), cudaMemcpyDeviceToHost));
        } else {
            CK(cudaMemcpy2D(w, L.kp * sizeof(float), host, K * sizeof(float), K * sizeof(float), L.cout,
                            cudaMemcpyHostToDevice));
            CK(cudaMemcpy(b, host + (int64_t)L.cout * K, L.cout * sizeof(float), cudaMemcpyHostToDevice));
            f32_to_bf16_kernel<<<64, 256>>>(L.w, L.wb, (int64_t)L.cout * L.kp);
            CK(cudaGetLastError());
            FG_LEGACY_FENCE();
        }
        host += (int64_t)L.cout * K + L.cout;
    }
    CK(cudaDeviceSynchronize());
    return FG_OK;
}

// input [B][Z][Y][X][2] FP32 (device or host) -> network input buffer
static int unet_load_input(fg_unet *u, const float *in, int mem) {
    UnetBufs &b = u->buf;
    const int64_t nv = b.v0.nvox();
    const float *src = in;
    float *tmp = nullptr;
    if (mem == FG_HOST) {
        CK(cudaMalloc(&tmp, nv * 2 * sizeof(float)));
        CK(cudaMemcpyAsync(tmp, in, nv * 2 * sizeof(float), cudaMemcpyHostToDevice, u->stream));
        src = tmp;
    }
    int blocks;
    grid_launch(nv, blocks);
    f32x2_to_x0_kernel<<<blocks, 256, 0, u->stream>>>(src, nv, TView{b.x0, 2, 0});
    CK(cudaGetLastError());
    if (tmp) {
        CK(cudaStreamSynchronize(u->stream));
        cudaFree(tmp);
    }
    return FG_OK;
}

static int unet_load_target(fg_unet *u, const float *t, int mem) {
    const int64_t nv = u->buf.v0.nvox();
    CK(cudaMemcpyAsync(u->buf.target, t, nv * sizeof(float),
                       mem == FG_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, u->stream));
    return FG_OK;
}

// forward + loss + backward; loss on the host (block partials summed in order)
static int unet_loss_grad(fg_unet *u, float *loss) {
    UnetBufs &b = u->buf;
    int rc;
    if ((rc = unet_forward(u))) return rc;
    const int64_t nv = b.v0.nvox();
    const int blocks = (int)std::min<int64_t>((nv + 255) / 256, 1024);
    mse_kernel<<<blocks, 256, 0, u->stream>>>(TView{b.out, 8, 0}, b.target, nv, 8, TView{b.dout, 8, 0}, b.msep);
    CK(cudaGetLastError());
    if ((rc = unet_backward(u))) return rc;
    std::vector<float> part(blocks);
    CK(cudaMemcpyAsync(part.data(), b.msep, blocks * sizeof(float), cudaMemcpyDeviceToHost, u->stream));
    CK(cudaStreamSynchronize(u->stream));
    double s = 0.0;
    for (float v : part) s += v;
    if (loss) *loss = (float)(s / (double)nv);
    return FG_OK;
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8) on the gradients in gw/gb
static int unet_adam(fg_unet *u, float lr) {
    u->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.f - std::pow(b1, (float)u->step), bc2 = 1.f - std::pow(b2, (float)u->step);
    for (auto &L : u->L) {
        const int nw = L.cout * L.kp;
        adam_kernel<<<64, 256, 0, u->stream>>>(L.w, L.gw, L.mw, L.vw, nw, lr, b1, b2, 1e-8f, bc1, bc2, L.wb);
        adam_kernel<<<1, 64, 0, u->stream>>>(L.b, L.gb, L.mb, L.vb, L.cout, lr, b1, b2, 1e-8f, bc1, bc2, nullptr);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(u->stream));
    return FG_OK;
}

// Reads (and clears) the network's own device error word after a synchronised call.
static int unet_check_err(fg_unet *u) {
    int h = 0;
    CK(cudaMemcpy(&h, u->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        CK(cudaMemset(u->d_err, 0, sizeof(int)));
        return fail(FG_DEVICE_TIMEOUT, "device-side wait timed out in the network's convolution");
    }
    return FG_OK;
}

extern "C" {

FG_API int fg_unet_create(const int channels[3], uint64_t seed, fg_unet **out) {
    if (!out) return fail(FG_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int c[3] = {16, 32, 48};
    if (channels)
        for (int i = 0; i < 3; ++i) c[i] = channels[i];
    const int allowed[] = {8, 16, 32, 48, 64};
    for (int i = 0; i < 3; ++i)
        if (std::find(std::begin(allowed), std::end(allowed), c[i]) == std::end(allowed))
            return fail(FG_UNSUPPORTED, "channel count %d not supported (8, 16, 32, 48, 64)", c[i]);
    if (c[1] + c[0] > 80 || c[2] + c[1] > 80 + 32)
        return fail(FG_UNSUPPORTED, "channel counts too large");
    fg_unet *u = new fg_unet();
    CK(cudaGetDevice(&u->device));
    u->C0 = c[0]; u->C1 = c[1]; u->C2 = c[2];
    if (const char *e = std::getenv("FG_UNET_TC")) u->tc = std::atoi(e) != 0;
    if (cudaMalloc(&u->d_err, sizeof(int)) != cudaSuccess || cudaMemset(u->d_err, 0, sizeof(int)) != cudaSuccess ||
        conv_tc_init() != FG_OK) {
        fg_unet_destroy(u);
        return fail(FG_CUDA_ERROR, "network set-up failed");
    }
    u->err = u->d_err;
    const int cin[NLAYERS] = {2, c[0], c[0], c[1], c[1], c[2], c[2] + c[1], c[1] + c[0], c[0]};
    const int cout[NLAYERS] = {c[0], c[0], c[1], c[1], c[2], c[2], c[1], c[0], 8};
    for (int l = 0; l < NLAYERS; ++l) {
        int rc = unet_layer_alloc(u->L[l], cin[l], cout[l], seed * 16 + l);
        if (rc) { fg_unet_destroy(u); return rc; }
    }
    CK(cudaDeviceSynchronize());
    *out = u;
    return FG_OK;
}

FG_API void fg_unet_destroy(fg_unet *u) {
    if (!u) return;
    cudaSetDevice(u->device);
    cudaDeviceSynchronize();
    for (auto &L : u->L) {
        void *p[] = {L.w, L.b, L.wb, L.gw, L.gb, L.mw, L.vw, L.mb, L.vb};
        for (void *q : p) if (q) cudaFree(q);
    }
    unet_free_bufs(u->buf);
    if (u->wflip) cudaFree(u->wflip);
    if (u->d_err) cudaFree(u->d_err);
    delete u;
}

FG_API int64_t fg_unet_num_params(const fg_unet *u) {
    if (!u) return -1;
    std::vector<int64_t> o;
    unet_params_layout(u, &o);
    return o.back();
}

FG_API int fg_unet_get_params(fg_unet *u, float *host) {
    if (!u || !host) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    CK(cudaSetDevice(u->device));
    return unet_copy_params(u, host, true, false);
}

FG_API int fg_unet_set_params(fg_unet *u, const float *host) {
    if (!u || !host) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    CK(cudaSetDevice(u->device));
    return unet_copy_params(u, const_cast<float *>(host), false, false);
}

FG_API int fg_unet_get_grads(fg_unet *u, float *host) {
    if (!u || !host) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    CK(cudaSetDevice(u->device));
    return unet_copy_params(u, host, true, true);
}

FG_API int fg_unet_forward(fg_unet *u, const float *in, int B, int Z, int Y, int X, float *out, int mem) {
    if (!u || !in || !out || B < 1) return fail(FG_INVALID_ARGUMENT, "bad arguments");
    CK(cudaSetDevice(u->device));
    u->stream = nullptr;
    u->err = u->d_err;
    int rc;
    if ((rc = unet_ensure_bufs(u, B, Z, Y, X)) || (rc = unet_load_input(u, in, mem)) || (rc = unet_forward(u)))
        return rc;
    const int64_t nv = u->buf.v0.nvox();
    float *dst = out, *tmp = nullptr;
    if (mem == FG_HOST) { CK(cudaMalloc(&tmp, nv * sizeof(float))); dst = tmp; }
    int blocks;
    grid_launch(nv, blocks);
    out0_to_f32_kernel<<<blocks, 256, 0, u->stream>>>(TView{u->buf.out, 8, 0}, nv, dst);
    CK(cudaGetLastError());
    if (tmp) {
        CK(cudaMemcpy(out, tmp, nv * sizeof(float), cudaMemcpyDeviceToHost));
        cudaFree(tmp);
    }
    CK(cudaDeviceSynchronize());
    return unet_check_err(u);
}

// Loss and gradients of the mean squared error between output channel 0 and
// target (no parameter update); fg_unet_get_grads reads them.
FG_API int fg_unet_loss_grad(fg_unet *u, const float *in, const float *target, int B, int Z, int Y, int X,
                             float *loss, int mem) {
    if (!u || !in || !target || B < 1) return fail(FG_INVALID_ARGUMENT, "bad arguments");
    CK(cudaSetDevice(u->device));
    u->stream = nullptr;
    u->err = u->d_err;
    int rc;
    if ((rc = unet_ensure_bufs(u, B, Z, Y, X)) || (rc = unet_load_input(u, in, mem)) ||
        (rc = unet_load_target(u, target, mem)) || (rc = unet_loss_grad(u, loss)))
        return rc;
    CK(cudaDeviceSynchronize());
    return unet_check_err(u);
}

// One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the loss of the batch.
FG_API int fg_unet_train_step(fg_unet *u, const float *in, const float *target, int B, int Z, int Y, int X,
                              float lr, float *loss, int mem) {
    int rc;
    if ((rc = fg_unet_loss_grad(u, in, target, B, Z, Y, X, loss, mem))) return rc;
    return unet_adam(u, lr);
}

// Coarse log-kappa channel of the learned correction: kappa at the DOFs
// (plain layout, host), restricted `levels` times (1 to 4) to the network
// volume.  Every level's extents must be odd and the network volume's 1 mod 4
// and >= 5, so the DOF lattice's cell counts (p times the element counts) must
// be multiples of 4 * 2^levels.
FG_API int fg_op_set_nodal_kappa(fg_op *op, const double *kappa_nodal, int levels) {
    FG_NEED_BOX(op, "fg_op_set_nodal_kappa");
    if (!op || !kappa_nodal) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (levels < 1 || levels > 4) return fail(FG_INVALID_ARGUMENT, "levels must be 1 to 4");
    const int m = 4 << levels;
    const int cx = op->g.NI - 1, cy = op->g.NJ - 1, cz = op->g.NK - 1;
    if (cx % m || cy % m || cz % m || cx / m < 1 || cy / m < 1 || cz / m < 1)
        return fail(FG_UNSUPPORTED, "the learned correction needs DOF-lattice cell counts (p * elements) "
                                    "that are multiples of %d", m);
    if (op->Nn >= (int64_t)1 << 31) return fail(FG_UNSUPPORTED, "the learned correction needs < 2^31 DOFs");
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    int rc;
    if ((rc = ensure_solver_buffers(op))) return rc;
    if (op->nn_lk && op->nn_levels != levels) {
        float *bufs[] = {op->nn_lk, op->nn_rc, op->nn_oc};
        for (float *b : bufs) cudaFree(b);
        for (float *t : op->nn_tmp) cudaFree(t);
        op->nn_tmp.clear();
        op->nn_lk = op->nn_rc = op->nn_oc = nullptr;
    }
    op->nn_levels = levels;
    const Vol Vc = nn_coarse_vol(op);
    const int64_t nv = Vc.nvox();
    if (!op->nn_lk) {
        CK(cudaMalloc(&op->nn_lk, nv * sizeof(float)));
        CK(cudaMalloc(&op->nn_rc, nv * sizeof(float)));
        CK(cudaMalloc(&op->nn_oc, nv * sizeof(float)));
        for (int l = 1; l < levels; ++l) {
            float *t = nullptr;
            CK(cudaMalloc(&t, nn_vol(op, l).nvox() * sizeof(float)));
            op->nn_tmp.push_back(t);
        }
        if (!op->nn_scale) CK(cudaMalloc(&op->nn_scale, 4 * sizeof(double)));
    }
    std::vector<double> lg(op->N);
    for (int64_t i = 0; i < op->N; ++i) lg[i] = std::log(std::max(kappa_nodal[i], 1e-300));
    if ((rc = to_native(op, op->cd, lg.data(), FG_HOST))) return rc;
    // full weighting averages (its weights sum to 1 away from the boundary)
    if ((rc = nn_restrict<double>(op, op->cd, op->nn_lk))) return rc;
    CK(cudaStreamSynchronize(op->stream));
    return FG_OK;
}

FG_API int fg_op_attach_unet(fg_op *op, fg_unet *net) {
    FG_NEED_BOX(op, "fg_op_attach_unet");
    if (!op) return fail(FG_INVALID_ARGUMENT, "NULL op");
    std::lock_guard<std::mutex> lk(op->mu);
    if (net && net->device != op->device) return fail(FG_INVALID_ARGUMENT, "network on another device");
    op->nn = net;
    op->nn_times.clear();
    return FG_OK;
}

// Training pairs from a plain Chebyshev-PCG solve of A x = b (x0 = 0): at
// iterations 0, every, 2*every, ... the iterate x_k gives
//   input  [Zc][Yc][Xc][2] = (R (b - A x_k) / s_k, R log kappa),
//   target [Zc][Yc][Xc]    = (x* - x_k) at the coarse vertices / s_k,
// s_k = rms(R (b - A x_k)); device FP32 outputs, up to max_pairs.
FG_API int fg_op_collect_pairs(fg_op *op, const double *b, const fg_cfg *cfg_in, int every, int max_pairs,
                               float *d_in, float *d_target, int *n_pairs) {
    FG_NEED_BOX(op, "fg_op_collect_pairs");
    if (!op || !b || !d_in || !d_target || !n_pairs || every < 1 || max_pairs < 1)
        return fail(FG_INVALID_ARGUMENT, "bad arguments");
    if (!op->nn_lk) return fail(FG_INVALID_ARGUMENT, "call fg_op_set_nodal_kappa first");
    fg_cfg cfg;
    if (cfg_in) cfg = *cfg_in; else fg_cfg_default(&cfg);
    cfg.precision = FG_FP64;
    cfg.precond = FG_PC_CHEBYSHEV;
    cfg.check_interval = every;
    int rc;
    if ((rc = validate_cfg(cfg))) return rc;
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    if ((rc = ensure_solver_buffers(op)) || (rc = ensure_dinv(op))) return rc;
    if (!op->have_lmax) {
        if ((rc = estimate_lmax(op, cfg.power_iters > 0 ? cfg.power_iters : 20, &op->lmax_est))) return rc;
        op->have_lmax = true;
    }
    const double lmax = (cfg.lmax_safety > 0 ? cfg.lmax_safety : 1.1) * op->lmax_est;
    const ChebCoef cc = cheb_coefs(lmax / (cfg.lmin_ratio > 0 ? cfg.lmin_ratio : 30.0), lmax, cfg.cheb_degree);
    const int64_t n = op->Nn;
    std::vector<double *> stash;
    auto cleanup = [&]() { for (double *p : stash) cudaFree(p); };
    struct G { std::function<void()> f; ~G() { f(); } } guard{cleanup};
    auto push = [&]() -> int {
        if ((int)stash.size() >= max_pairs) return FG_OK;
        double *p = nullptr;
        CK(cudaMalloc(&p, n * sizeof(double)));
        CK(cudaMemcpyAsync(p, op->xw, n * sizeof(double), cudaMemcpyDeviceToDevice, op->stream));
        stash.push_back(p);
        return FG_OK;
    };
    if ((rc = to_native(op, op->bw, b, FG_HOST))) return rc;
    CK(cudaMemsetAsync(op->xw, 0, n * sizeof(double), op->stream));
    if ((rc = push())) return rc;
    PcgBufs<double> B{op->qd, op->face, op->dinv, op->xw, op->bw, op->r, op->z, op->pv, op->ap,
                      op->cres, op->cd, op->ct, op->st};
    set_state(op, op->st, cfg.rtol, cfg.atol, cfg.max_iter);
    SolverState h{};
    int64_t applies = 0;
    if ((rc = pcg_run<double>(op, B, false, &cc, cfg.max_iter, every, false, &h, &applies,
                              [&](int) { return push(); })))
        return rc;
    Grid g = op->g;
    g.ess = op->ess_tags;
    const Vol Vc = nn_coarse_vol(op);
    const int64_t nv = Vc.nvox();
    int blocks;
    grid_launch(nv, blocks);
    for (size_t j = 0; j < stash.size(); ++j) {
        if ((rc = apply_native(op, stash[j], op->ap, 0, 1, nullptr))) return rc;
        k_lincomb2<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->r, 1.0, op->bw, -1.0, op->ap);
        if ((rc = nn_restrict<double>(op, op->r, op->nn_rc))) return rc;
        rms_kernel<<<1, 1024, 0, op->stream>>>(op->nn_rc, nv, op->nn_scale);
        pack_input_f32_kernel<<<blocks, 256, 0, op->stream>>>(op->nn_rc, op->nn_lk, nv, op->nn_scale,
                                                              d_in + (int64_t)j * nv * 2);
        pair_target_kernel<<<blocks, 256, 0, op->stream>>>(g, op->xw, stash[j], Vc, 1 << op->nn_levels, op->nn_scale,
                                                           d_target + (int64_t)j * nv);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(op->stream));
    *n_pairs = (int)stash.size();
    return check_device_error(op);
}

// Residuals of a plain Chebyshev-PCG solve of A x = b (x0 = 0) at iterations
// 0, every, 2*every, ...: up to max_res native-layout FP64 vectors written to
// d_out ([max_res][fg_op_native_len], device); the count in *n_res.
FG_API int fg_op_collect_residuals(fg_op *op, const double *b, const fg_cfg *cfg_in, int every, int max_res,
                                   double *d_out, int *n_res) {
    FG_NEED_BOX(op, "fg_op_collect_residuals");
    if (!op || !b || !d_out || !n_res || every < 1 || max_res < 1)
        return fail(FG_INVALID_ARGUMENT, "bad arguments");
    fg_cfg cfg;
    if (cfg_in) cfg = *cfg_in; else fg_cfg_default(&cfg);
    cfg.precision = FG_FP64;
    cfg.precond = FG_PC_CHEBYSHEV;
    cfg.check_interval = every;
    int rc;
    if ((rc = validate_cfg(cfg))) return rc;
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    if ((rc = ensure_solver_buffers(op)) || (rc = ensure_dinv(op))) return rc;
    if (!op->have_lmax) {
        if ((rc = estimate_lmax(op, cfg.power_iters > 0 ? cfg.power_iters : 20, &op->lmax_est))) return rc;
        op->have_lmax = true;
    }
    const double lmax = (cfg.lmax_safety > 0 ? cfg.lmax_safety : 1.1) * op->lmax_est;
    const ChebCoef cc = cheb_coefs(lmax / (cfg.lmin_ratio > 0 ? cfg.lmin_ratio : 30.0), lmax, cfg.cheb_degree);
    const int64_t n = op->Nn;
    int count = 0;
    auto push = [&]() -> int {
        if (count >= max_res) return FG_OK;
        CK(cudaMemcpyAsync(d_out + (int64_t)count * n, op->r, n * sizeof(double), cudaMemcpyDeviceToDevice,
                           op->stream));
        ++count;
        return FG_OK;
    };
    if ((rc = to_native(op, op->bw, b, FG_HOST))) return rc;
    CK(cudaMemsetAsync(op->xw, 0, n * sizeof(double), op->stream));
    CK(cudaMemcpyAsync(op->r, op->bw, n * sizeof(double), cudaMemcpyDeviceToDevice, op->stream));
    if ((rc = push())) return rc;
    PcgBufs<double> B{op->qd, op->face, op->dinv, op->xw, op->bw, op->r, op->z, op->pv, op->ap,
                      op->cres, op->cd, op->ct, op->st};
    set_state(op, op->st, cfg.rtol, cfg.atol, cfg.max_iter);
    SolverState h{};
    int64_t applies = 0;
    if ((rc = pcg_run<double>(op, B, false, &cc, cfg.max_iter, every, false, &h, &applies,
                              [&](int) { return push(); })))
        return rc;
    CK(cudaStreamSynchronize(op->stream));
    *n_res = count;
    return check_device_error(op);
}

// One Adam step of the learned coarse correction on the energy loss of B
// residuals r_b (device, native layout, [B][fg_op_native_len] FP64, zero on
// essential DOFs).  Per sample, with s = rms(R^L r) and network output n,
//   c = s 8^L P^L n  (zero on essential DOFs),
//   loss_b = (1/2 c.Ac - c.r) / (s^2 64^L Nc),   Nc = network voxels,
// whose minimiser over c in range(P^L) is the Galerkin coarse correction;
// d loss_b / d n = R^L (A c - r) / (s Nc)  (P^T = 8 R per level).  The
// reported loss is the batch mean.
FG_API int fg_unet_train_energy(fg_unet *u, fg_op *op, const double *d_res, int B, float lr, float *loss) {
    FG_NEED_BOX(op, "fg_unet_train_energy");
    if (!u || !op || !d_res || B < 1) return fail(FG_INVALID_ARGUMENT, "bad arguments");
    if (!op->nn_lk) return fail(FG_INVALID_ARGUMENT, "call fg_op_set_nodal_kappa first");
    if (u->device != op->device) return fail(FG_INVALID_ARGUMENT, "network on another device");
    std::lock_guard<std::mutex> lk(op->mu);
    CK(cudaSetDevice(op->device));
    int rc;
    if ((rc = ensure_solver_buffers(op))) return rc;
    u->stream = op->stream;
    u->err = op->d_err;
    const Vol Vc = nn_coarse_vol(op);
    if ((rc = unet_ensure_bufs(u, B, Vc.Z, Vc.Y, Vc.X))) return rc;
    const int64_t nv = Vc.nvox(), n = op->Nn;
    double *tb = nullptr;  // per sample: s, c.Ac, c.r
    CK(cudaMalloc(&tb, (size_t)B * 4 * sizeof(double)));
    struct Free { double *p; ~Free() { cudaFree(p); } } fr{tb};
    int blocks;
    grid_launch(nv, blocks);
    UnetBufs &ub = u->buf;
    for (int b = 0; b < B; ++b) {
        if ((rc = nn_restrict<double>(op, d_res + (int64_t)b * n, op->nn_rc))) return rc;
        rms_kernel<<<1, 1024, 0, op->stream>>>(op->nn_rc, nv, tb + 4 * b);
        pack_input_kernel<<<blocks, 256, 0, op->stream>>>(op->nn_rc, op->nn_lk, nv, tb + 4 * b,
                                                          TView{ub.x0 + (int64_t)b * nv * 2, 2, 0});
    }
    CK(cudaGetLastError());
    if ((rc = unet_forward(u))) return rc;
    const float coef = (float)(1.0 / ((double)nv * B));
    const double mult = nn_mult(op);
    for (int b = 0; b < B; ++b) {
        const double *r = d_res + (int64_t)b * n;
        out0_to_f32_kernel<<<blocks, 256, 0, op->stream>>>(TView{ub.out + (int64_t)b * nv * 8, 8, 0}, nv,
                                                           op->nn_oc);
        if ((rc = nn_prolong<double>(op, op->nn_oc, op->pv, tb + 4 * b, mult, 0))) return rc;
        if ((rc = apply_native(op, op->pv, op->ap, 0, 1, nullptr))) return rc;
        k_energy_terms<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(n, op->pv, op->ap, r, op->partials, op->st);
        CK(cudaMemcpyAsync(tb + 4 * b + 1, &op->st->tmp[0], 2 * sizeof(double), cudaMemcpyDeviceToDevice,
                           op->stream));
        if ((rc = nn_restrict<double>(op, op->ap, op->nn_rc))) return rc;
        energy_grad_kernel<<<blocks, 256, 0, op->stream>>>(op->nn_rc, nv, coef, tb + 4 * b,
                                                           TView{ub.dout + (int64_t)b * nv * 8, 8, 0});
        CK(cudaGetLastError());
    }
    if ((rc = unet_backward(u))) return rc;
    if ((rc = unet_adam(u, lr))) return rc;
    std::vector<double> h((size_t)B * 4);
    CK(cudaMemcpy(h.data(), tb, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
    double L = 0.0;
    for (int b = 0; b < B; ++b) {
        const double sc = h[4 * b] > 0.0 ? h[4 * b] : 1.0;
        L += (0.5 * h[4 * b + 1] - h[4 * b + 2]) / (sc * sc * mult * mult * (double)nv);
    }
    if (loss) *loss = (float)(L / B);
    return check_device_error(op);
}

// ---------------------------------------------------------------------------
// Linear forms, L2 error and lumped mass (one-time work around the solve).
// ---------------------------------------------------------------------------
}  // extern "C"

// n-point Gauss-Legendre rule on [-1, 1]: closed forms up to 4 points (the
// operator's rules), Newton on the Legendre recurrence above
static void gauss_rule(int n, double *x, double *w) {
    if (n <= 4) {
        gauss_legendre(n, x, w);
        return;
    }
    for (int i = 0; i < n; ++i) {
        double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        x[n - 1 - i] = z;
        w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

struct FormSetup {
    FormArgs A{};
    double *d_vc = nullptr;
    int64_t E = 0, N = 0;
    ~FormSetup() {
        if (d_vc) cudaFree(d_vc);
    }
};

static int form_setup(const fg_mesh *mesh, int order, int nq, FormSetup &F) {
    if (!mesh) return fail(FG_INVALID_ARGUMENT, "NULL mesh");
    if (mesh->nx < 1 || mesh->ny < 1 || mesh->nz < 1) return fail(FG_INVALID_ARGUMENT, "empty mesh");
    if (order < 1 || order > FG_MAXP) return fail(FG_UNSUPPORTED, "order %d not supported (1..%d)", order, FG_MAXP);
    if (nq < 1 || nq > FORM_MAXQ) return fail(FG_UNSUPPORTED, "%d quadrature points not supported (1..%d)", nq, FORM_MAXQ);
    Grid &g = F.A.g;
    g.nx = mesh->nx; g.ny = mesh->ny; g.nz = mesh->nz; g.p = order;
    g.NI = mesh->nx * order + 1; g.NJ = mesh->ny * order + 1; g.NK = mesh->nz * order + 1;
    F.E = (int64_t)g.nx * g.ny * g.nz;
    F.N = (int64_t)g.NI * g.NJ * g.NK;
    F.A.nq = nq;
    gauss_rule(nq, F.A.gx, F.A.gw);
    for (int q = 0; q < nq; ++q) {
        double phi[FG_MAXP + 1], dphi[FG_MAXP + 1];
        lagrange1d(order, F.A.gx[q], phi, dphi);
        for (int d = 0; d <= order; ++d) F.A.B[q][d] = phi[d];
    }
    if (mesh->vcoord) {
        const size_t nb = sizeof(double) * 3 * (size_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
        CK(cudaMalloc(&F.d_vc, nb));
        CK(cudaMemcpy(F.d_vc, mesh->vcoord, nb, cudaMemcpyDefault));
        FG_LEGACY_FENCE();
    }
    F.A.vcoord = F.d_vc;
    return FG_OK;
}

// device copy of n doubles from host or device memory (owned = allocated here)
struct DevBuf {
    double *p = nullptr;
    bool owned = false;
    ~DevBuf() {
        if (owned && p) cudaFree(p);
    }
};
static int dev_in(const double *src, int64_t n, int mem, DevBuf &d) {
    if (!src) return FG_OK;
    if (mem == FG_DEVICE) {
        d.p = const_cast<double *>(src);
        return FG_OK;
    }
    CK(cudaMalloc(&d.p, sizeof(double) * (size_t)std::max<int64_t>(n, 1)));
    d.owned = true;
    CK(cudaMemcpy(d.p, src, sizeof(double) * n, cudaMemcpyHostToDevice));
    FG_LEGACY_FENCE();
    return FG_OK;
}

// out = M_f 1 with M_f the mass form of the coefficient f (sum_j phi_j = 1),
// then the essential rows of ess_tags set to zero
static int mass_times_ones(const fg_mesh *mesh, int order, const double *f_q, double f_const, int ess_tags,
                           double *out, int mem) {
    fg_op *op = nullptr;
    int rc = fg_op_create(mesh, order, order + 1, FG_MASS, 1.0, 0.0, nullptr, 0.0, f_q, f_const, 0, &op);
    if (rc) return rc;
    struct Kill { fg_op *o; ~Kill() { fg_op_destroy(o); } } kill{op};
    std::lock_guard<std::mutex> lk(op->mu);
    double *ones = nullptr, *y = nullptr;
    CK(cudaMalloc(&ones, sizeof(double) * op->Nn));
    struct F1 { double *p; ~F1() { cudaFree(p); } } f1{ones};
    CK(cudaMalloc(&y, sizeof(double) * op->Nn));
    struct F2 { double *p; ~F2() { cudaFree(p); } } f2{y};
    CK(cudaMemsetAsync(ones, 0, sizeof(double) * op->Nn, op->stream));
    k_invert_diag<double><<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(op->g, ones, ones);  // 1 on DOFs, 0 on pads
    CK(cudaGetLastError());
    if ((rc = apply_native(op, ones, y, 0, 0, nullptr))) return rc;
    if (ess_tags) {
        Grid g = op->g;
        g.ess = ess_tags;
        zero_ess_kernel<<<VEC_GRID, VEC_THREADS, 0, op->stream>>>(g, y);
        CK(cudaGetLastError());
    }
    if ((rc = from_native(op, out, y, mem))) return rc;
    CK(cudaStreamSynchronize(op->stream));
    return check_device_error(op);
}

extern "C" {

FG_API int fg_quadrature_points(const fg_mesh *mesh, int nq, double *xyz, int mem) {
    if (!xyz) return fail(FG_INVALID_ARGUMENT, "NULL output");
    if (mem != FG_HOST && mem != FG_DEVICE) return fail(FG_INVALID_ARGUMENT, "bad mem %d", mem);
    FormSetup F;
    int rc;
    if ((rc = form_setup(mesh, 1, nq, F))) return rc;
    const int Q3 = nq * nq * nq;
    const int64_t n = F.E * Q3 * 3;
    double *out = xyz;
    if (mem == FG_HOST) CK(cudaMalloc(&out, sizeof(double) * n));
    struct F1 { double *p; bool own; ~F1() { if (own) cudaFree(p); } } f1{out, mem == FG_HOST};
    qp_coords_kernel<<<VEC_GRID * 4, 256>>>(F.A, out);
    CK(cudaGetLastError());
    if (mem == FG_HOST) CK(cudaMemcpy(xyz, out, sizeof(double) * n, cudaMemcpyDeviceToHost));
    CK(cudaDeviceSynchronize());
    return FG_OK;
}

FG_API int fg_assemble_source(const fg_mesh *mesh, int order, const double *f_q, double f_const, int ess_tags,
                              double *b, int mem) {
    if (!b) return fail(FG_INVALID_ARGUMENT, "NULL output");
    if (mem != FG_HOST && mem != FG_DEVICE) return fail(FG_INVALID_ARGUMENT, "bad mem %d", mem);
    if (ess_tags < 0 || ess_tags > 63) return fail(FG_INVALID_ARGUMENT, "bad ess_tags %d", ess_tags);
    return mass_times_ones(mesh, order, f_q, f_const, ess_tags, b, mem);
}

FG_API int fg_lumped_mass(const fg_mesh *mesh, int order, const double *rho_q, double rho_const, double *diag,
                          int mem) {
    if (!diag) return fail(FG_INVALID_ARGUMENT, "NULL output");
    if (mem != FG_HOST && mem != FG_DEVICE) return fail(FG_INVALID_ARGUMENT, "bad mem %d", mem);
    return mass_times_ones(mesh, order, rho_q, rho_const, 0, diag, mem);
}

FG_API int fg_lumped_apply(const double *diag, const double *x, double *y, int64_t n, int mode, int mem) {
    if (!diag || !x || !y || n < 0) return fail(FG_INVALID_ARGUMENT, "bad arguments");
    if (mode < 0 || mode > 2) return fail(FG_INVALID_ARGUMENT, "bad mode %d", mode);
    if (mem != FG_HOST && mem != FG_DEVICE) return fail(FG_INVALID_ARGUMENT, "bad mem %d", mem);
    if (n == 0) return FG_OK;
    DevBuf dd, dx, dy;
    int rc;
    if ((rc = dev_in(diag, n, mem, dd)) || (rc = dev_in(x, n, mem, dx)) || (rc = dev_in(y, n, mem, dy))) return rc;
    lumped_apply_kernel<<<VEC_GRID, 256>>>(dd.p, dx.p, dy.p, n, mode);
    CK(cudaGetLastError());
    if (mem == FG_HOST) CK(cudaMemcpy(y, dy.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    CK(cudaDeviceSynchronize());
    return FG_OK;
}

FG_API int fg_l2_error(const fg_mesh *mesh, int order, int nq, const double *u, const double *u_q, double *err,
                       int mem) {
    if (!u || !err) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (mem != FG_HOST && mem != FG_DEVICE) return fail(FG_INVALID_ARGUMENT, "bad mem %d", mem);
    FormSetup F;
    int rc;
    if ((rc = form_setup(mesh, order, nq, F))) return rc;
    DevBuf du, duq;
    if ((rc = dev_in(u, F.N, mem, du)) || (rc = dev_in(u_q, F.E * nq * nq * nq, mem, duq))) return rc;
    double *part = nullptr;
    CK(cudaMalloc(&part, sizeof(double) * VEC_GRID));
    struct F1 { double *p; ~F1() { cudaFree(p); } } f1{part};
    l2_error_kernel<<<VEC_GRID, 256>>>(F.A, du.p, duq.p, part);
    CK(cudaGetLastError());
    std::vector<double> h(VEC_GRID);
    CK(cudaMemcpy(h.data(), part, sizeof(double) * VEC_GRID, cudaMemcpyDeviceToHost));
    double s = 0.0;
    for (double v : h) s += v;  // block order: deterministic
    *err = std::sqrt(s);
    return FG_OK;
}

// ---------------------------------------------------------------------------
// Tetrahedral PA operator (TetP1 / TetP2 on unstructured Tet4 meshes)
// ---------------------------------------------------------------------------
FG_API int fg_tet_create(int order, int64_t n_nodes, const double *coords, int64_t n_elem, const int32_t *elem_dofs,
                         int64_t n_dofs, int kind, double c_mass, double c_diff, const double *kappa_q,
                         double kappa_const, const double *rho_q, double rho_const, int quad_order,
                         const uint8_t *ess, fg_tet **out) {
    if (!out) return fail(FG_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (order < 1 || order > 3) return fail(FG_UNSUPPORTED, "tet order %d not supported (1..3)", order);
    if (kind < 1 || kind > 3) return fail(FG_INVALID_ARGUMENT, "bad operator kind %d", kind);
    if (!coords || !elem_dofs || n_nodes < 4 || n_elem < 1 || n_dofs < n_nodes || n_dofs >= ((int64_t)1 << 31))
        return fail(FG_INVALID_ARGUMENT, "bad tet mesh arguments");
    if (n_elem * (order == 1 ? 4 : (order == 2 ? 10 : 20)) >= ((int64_t)1 << 31))
        return fail(FG_UNSUPPORTED, "too many elements for 32-bit element-local slots");
    int rc;
    fg_tet *t = new fg_tet();
    struct Bail { fg_tet *t; bool armed = true; ~Bail() { if (armed) tet_free(t); } } bail{t};
    CK(cudaGetDevice(&t->device));
    t->p = order;
    t->nl = order == 1 ? 4 : (order == 2 ? 10 : 20);
    t->kind = kind;
    t->E = n_elem;
    t->N = n_dofs;
    t->n_nodes = n_nodes;
    const int nl = t->nl;
    CK(cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking));
    CK(cudaMalloc(&t->d_err, sizeof(int)));
    CK(cudaMemset(t->d_err, 0, sizeof(int)));
    FG_LEGACY_FENCE();
    // element map: validate, transpose to [nl][E]; chunk order and chunk DOF lists
    std::vector<int32_t> h(n_elem * nl);
    CK(cudaMemcpy(h.data(), elem_dofs, sizeof(int32_t) * h.size(), cudaMemcpyDefault));
    std::vector<double> hc((size_t)n_nodes * 3);
    CK(cudaMemcpy(hc.data(), coords, sizeof(double) * hc.size(), cudaMemcpyDefault));
    std::vector<int32_t> soa(h.size());
    for (int64_t e = 0; e < n_elem; ++e)
        for (int i = 0; i < nl; ++i) {
            const int32_t d = h[e * nl + i];
            if (d < 0 || d >= n_dofs || (i < 4 && d >= n_nodes))
                return fail(FG_BOUNDS, "element %lld local DOF %d out of range", (long long)e, i);
            soa[(int64_t)i * n_elem + e] = d;
        }
    t->CE = order == 3 ? 256 : 512;
    if (const char *ev = std::getenv("FG_TET_CHUNK")) {
        const int v = std::atoi(ev);
        if (v >= 32 && v <= 1024 && v * nl <= 65536) t->CE = v;
    }
    if (const char *ev = std::getenv("FG_TET_WIDE")) t->wide = std::atoi(ev) != 0;
    ChunkPlan plan;
    std::vector<int32_t> perm;
    tet_plan_chunks(h, hc, n_elem, n_dofs, nl, t->CE, perm, plan);
    t->n_chunks = (int)plan.n_chunks;
    t->max_nu = plan.max_nu;
    if (tet_chunk_smem(nl, t->CE, t->max_nu) > 227 * 1024)
        return fail(FG_UNSUPPORTED, "tet chunk of %d elements needs too much shared memory", t->CE);
    t->n_shared = (int64_t)plan.sh_dof.size();
    t->n_part = plan.n_part;
    if ((rc = tet_upload(&t->dofs, soa.data(), soa.size())) ||
        (rc = tet_upload(&t->cu_slots, plan.cu_slots.data(), plan.cu_slots.size())) ||
        (rc = tet_upload(&t->cu_off, plan.cu_off.data(), plan.cu_off.size())) ||
        (rc = tet_upload(&t->cu_dof, plan.cu_dof.data(), plan.cu_dof.size())) ||
        (rc = tet_upload(&t->cu_pid, plan.cu_pid.data(), plan.cu_pid.size())) ||
        (rc = tet_upload(&t->cu_soff, plan.cu_soff.data(), plan.cu_soff.size())) ||
        (rc = tet_upload(&t->sh_dof, plan.sh_dof.data(), plan.sh_dof.size())) ||
        (rc = tet_upload(&t->sh_off, plan.sh_off.data(), plan.sh_off.size())) ||
        (rc = tet_upload(&t->coords, coords, (size_t)n_nodes * 3)))
        return rc;
    CK(cudaMalloc(&t->part, sizeof(double) * std::max<int64_t>(t->n_part, 1)));
    {   // element map and essential local DOFs in the chunk order
        std::vector<int32_t> ed(h.size());
        std::vector<uint8_t> he;
        if (ess) {
            he.resize(n_dofs);
            CK(cudaMemcpy(he.data(), ess, n_dofs, cudaMemcpyDefault));
        }
        std::vector<uint32_t> em(ess ? n_elem : 0, 0u);
        for (int64_t n = 0; n < n_elem; ++n) {
            const int64_t e = perm[n];
            for (int i = 0; i < nl; ++i) {
                const int32_t d = h[e * nl + i];
                ed[(int64_t)i * n_elem + n] = d;
                if (ess && he[d]) em[n] |= 1u << i;
            }
        }
        if ((rc = tet_upload(&t->edof, ed.data(), ed.size()))) return rc;
        if (ess && (rc = tet_upload(&t->emsk, em.data(), em.size()))) return rc;
    }
    if (ess && (rc = tet_upload(&t->ess, ess, (size_t)n_dofs))) return rc;
    // rule tables
    std::vector<double> pts, w;
    t->nq = tet_rule_host(quad_order, pts, w);
    if (t->nq > TET_MAXQ) return fail(FG_UNSUPPORTED, "quadrature order %d too high", quad_order);
    std::vector<double> phi((size_t)t->nq * nl), grad((size_t)t->nq * nl * 3);
    for (int q = 0; q < t->nq; ++q) tet_basis_host(order, &pts[3 * q], &phi[(size_t)q * nl], &grad[(size_t)q * nl * 3]);
    t->h_phi = phi;
    t->h_grad = grad;
    double *d_w = nullptr;
    if ((rc = tet_upload(&t->qp, pts.data(), pts.size())) || (rc = tet_upload(&t->phi, phi.data(), phi.size())) ||
        (rc = tet_upload(&t->grad, grad.data(), grad.size())) || (rc = tet_upload(&d_w, w.data(), w.size())))
        return rc;
    struct FW { double *p; ~FW() { cudaFree(p); } } fw{d_w};
    const double *d_kq = nullptr, *d_rq = nullptr;
    double *tk = nullptr, *tr = nullptr;
    struct FT { double **a, **b; ~FT() { if (*a) cudaFree(*a); if (*b) cudaFree(*b); } } ft{&tk, &tr};
    if (kappa_q) { if ((rc = tet_upload(&tk, kappa_q, (size_t)n_elem * t->nq))) return rc; d_kq = tk; }
    if (rho_q) { if ((rc = tet_upload(&tr, rho_q, (size_t)n_elem * t->nq))) return rc; d_rq = tr; }
    // geometry and point scalars in the caller's order, then the chunk order
    // and the diffusion moments (P1: S00 G, P2: 10)
    double *G0 = nullptr, *sk0 = nullptr, *sm0 = nullptr;
    int32_t *d_perm = nullptr;
    struct FS { double **a, **b, **c; int32_t **d;
        ~FS() { if (*a) cudaFree(*a); if (*b) cudaFree(*b); if (*c) cudaFree(*c); if (*d) cudaFree(*d); } }
        fs{&G0, &sk0, &sm0, &d_perm};
    CK(cudaMalloc(&G0, sizeof(double) * 6 * n_elem));
    CK(cudaMalloc(&t->G, sizeof(double) * 6 * n_elem));
    if (kind & 2) {
        CK(cudaMalloc(&sk0, sizeof(double) * t->nq * n_elem));
        CK(cudaMalloc(&t->sk, sizeof(double) * t->nq * n_elem));
    }
    if (kind & 1) {
        CK(cudaMalloc(&sm0, sizeof(double) * t->nq * n_elem));
        CK(cudaMalloc(&t->sm, sizeof(double) * t->nq * n_elem));
    }
    const int nmom = (kind & 2) ? (order == 1 ? 6 : (order == 2 ? 10 : 0)) : 0;
    if (nmom) CK(cudaMalloc(&t->Sm, sizeof(double) * nmom * n_elem));
    if ((rc = tet_upload(&d_perm, perm.data(), perm.size()))) return rc;
    TetArgs A = tet_args(t);
    A.G = G0;
    A.sk = sk0;
    A.sm = sm0;
    const int eb = (int)std::min<int64_t>((n_elem + 255) / 256, 148 * 16);
    tet_setup_kernel<<<eb, 256, 0, t->stream>>>(A, nl, t->coords, d_w, d_kq, kappa_const, d_rq, rho_const, c_mass,
                                                c_diff, G0, sk0, sm0, t->d_err);
    CK(cudaGetLastError());
    tet_permute_kernel<<<eb, 256, 0, t->stream>>>(n_elem, t->nq, kind, nmom, d_perm, t->qp, G0, sk0, sm0, t->G,
                                                  t->sk, t->sm, t->Sm);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(t->stream));
    int herr = 0;
    CK(cudaMemcpy(&herr, t->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) return fail(FG_BOUNDS, "degenerate tetrahedron (det J = 0)");
    bail.armed = false;
    *out = t;
    return FG_OK;
}

FG_API void fg_tet_destroy(fg_tet *t) { tet_free(t); }

FG_API int64_t fg_tet_ndofs(const fg_tet *t) { return t ? t->N : -1; }

FG_API int fg_tet_nq(const fg_tet *t) { return t ? t->nq : -1; }

FG_API int fg_tet_quadrature_points(fg_tet *t, double *xyz, int mem) {
    if (!t || !xyz) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (mem != FG_HOST && mem != FG_DEVICE) return fail(FG_INVALID_ARGUMENT, "bad mem %d", mem);
    std::lock_guard<std::mutex> lk(t->mu);
    CK(cudaSetDevice(t->device));
    const int64_t n = t->E * t->nq * 3;
    double *out = xyz;
    if (mem == FG_HOST) CK(cudaMalloc(&out, sizeof(double) * n));
    struct F1 { double *p; bool own; ~F1() { if (own) cudaFree(p); } } f1{out, mem == FG_HOST};
    const TetArgs A = tet_args(t);
    tet_qp_coords_kernel<<<VEC_GRID * 4, 256, 0, t->stream>>>(A, t->coords, t->qp, out);
    CK(cudaGetLastError());
    if (mem == FG_HOST) CK(cudaMemcpyAsync(xyz, out, sizeof(double) * n, cudaMemcpyDeviceToHost, t->stream));
    CK(cudaStreamSynchronize(t->stream));
    return FG_OK;
}

FG_API int fg_tet_apply(fg_tet *t, const double *x, double *y, int accumulate, int constrained, int mem) {
    if (!t || !x || !y) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (mem != FG_HOST && mem != FG_DEVICE) return fail(FG_INVALID_ARGUMENT, "bad mem %d", mem);
    if (constrained && !t->ess) return fail(FG_INVALID_ARGUMENT, "constrained apply needs the essential mask");
    std::lock_guard<std::mutex> lk(t->mu);
    CK(cudaSetDevice(t->device));
    const double *xd = x;
    double *yd = y;
    const size_t nb = sizeof(double) * t->N;
    if (mem == FG_HOST) {
        if (!t->xh) CK(cudaMalloc(&t->xh, nb));
        if (!t->yh) CK(cudaMalloc(&t->yh, nb));
        CK(cudaMemcpyAsync(t->xh, x, nb, cudaMemcpyHostToDevice, t->stream));
        if (accumulate) CK(cudaMemcpyAsync(t->yh, y, nb, cudaMemcpyHostToDevice, t->stream));
        xd = t->xh;
        yd = t->yh;
    }
    int rc;
    if ((rc = tet_launch_apply(t, xd, yd, accumulate, constrained, 0))) return rc;
    if (mem == FG_HOST) CK(cudaMemcpyAsync(y, yd, nb, cudaMemcpyDeviceToHost, t->stream));
    CK(cudaStreamSynchronize(t->stream));
    return FG_OK;
}

FG_API int fg_tet_apply_native(fg_tet *t, const double *x, double *y, int accumulate, int constrained) {
    if (!t || !x || !y) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (constrained && !t->ess) return fail(FG_INVALID_ARGUMENT, "constrained apply needs the essential mask");
    std::lock_guard<std::mutex> lk(t->mu);
    CK(cudaSetDevice(t->device));
    return tet_launch_apply(t, x, y, accumulate, constrained, 0);
}

FG_API int fg_tet_set_stream(fg_tet *t, void *stream) {
    if (!t) return fail(FG_INVALID_ARGUMENT, "NULL operator");
    std::lock_guard<std::mutex> lk(t->mu);
    CK(cudaSetDevice(t->device));
    CK(cudaStreamSynchronize(t->stream));
    if (t->own_stream) cudaStreamDestroy(t->stream);
    t->own_stream = false;
    t->stream = reinterpret_cast<cudaStream_t>(stream);
    return FG_OK;
}

FG_API int fg_tet_check(fg_tet *t) {
    if (!t) return fail(FG_INVALID_ARGUMENT, "NULL operator");
    std::lock_guard<std::mutex> lk(t->mu);
    CK(cudaSetDevice(t->device));
    CK(cudaStreamSynchronize(t->stream));
    return FG_OK;
}

FG_API int fg_tet_diagonal(fg_tet *t, double *d, int constrained, int mem) {
    if (!t || !d) return fail(FG_INVALID_ARGUMENT, "NULL argument");
    if (mem != FG_HOST && mem != FG_DEVICE) return fail(FG_INVALID_ARGUMENT, "bad mem %d", mem);
    if (constrained && !t->ess) return fail(FG_INVALID_ARGUMENT, "constrained diagonal needs the essential mask");
    std::lock_guard<std::mutex> lk(t->mu);
    CK(cudaSetDevice(t->device));
    double *dd = d;
    if (mem == FG_HOST) {
        if (!t->yh) CK(cudaMalloc(&t->yh, sizeof(double) * t->N));
        dd = t->yh;
    }
    int rc;
    if ((rc = tet_launch_apply(t, nullptr, dd, 0, constrained, 1))) return rc;
    if (mem == FG_HOST) CK(cudaMemcpyAsync(d, dd, sizeof(double) * t->N, cudaMemcpyDeviceToHost, t->stream));
    CK(cudaStreamSynchronize(t->stream));
    return FG_OK;
}

}  // extern "C"
