// pa_kernels.cuh -- partial-assembly (PA) mass / diffusion operator on a
// structured hex mesh of order P (Q = P+1 Gauss points per direction),
// hand-written for sm_100a.
//
// It computes the same operator as the reference's element loop
// (crates/assembly/src/partial.rs:85-130 mass, :154-208 diffusion, with the
// Hex8 isoparametric geometry of crates/assembly/src/assembler.rs:96-143),
// factored libCEED-style as E^T B^T D B E:
//   E    gather of the element DOFs from the L-vector (a TMA tile load of x),
//   B    sum-factorised interpolation / gradient to the quadrature points,
//   D    the quadrature data: 6 symmetric components w|detJ| kappa J^-1 J^-T
//        (diffusion) and/or w|detJ| rho (mass), precomputed once,
//   B^T  the transposed contractions,
//   E^T  a deterministic scatter with no floating-point atomics.
//
// Work decomposition.  A CTA owns an "item": a tile of 32 elements in x
// (one warp, one element per lane) by WY element rows in y (one warp per row),
// and sweeps TZ element layers in z.  Each thread keeps its element's
// contractions in registers.  Contributions of neighbouring elements to the
// DOFs they share are summed in a fixed order: across x by a warp shuffle,
// across y through shared memory between the row warps, across z by carrying
// the top DOF plane of a layer in shared memory into the next layer.  DOFs on
// the three upper faces of an item that belong to a neighbouring item are
// written to a per-item face buffer; fixup_kernel then adds them to the owner
// values in a fixed order.  The result is bit-identical from run to run.
//
// Streams into shared memory: the quadrature data of each warp is laid out in
// HBM in exactly the order the warp consumes it (one contiguous block per
// element column of quadrature points), and is streamed with 1-D bulk async
// copies (cp.async.bulk) into an S-deep ring of stages per warp.  The x tile
// of each layer is a 3-D TMA tensor load (cp.async.bulk.tensor, no multicast)
// into a double buffer.
#pragma once
#include <type_traits>
#include "fg_common.cuh"

#ifndef FG_Q3_QH  // Q3 FP64 full-format slab width in quadrature columns (Q: a whole qy slab)
#define FG_Q3_QH 2
#endif
#ifndef FG_Q3_NXB  // Q3 FP64 x tile buffers (1: single buffer, 3 CTAs per SM; 2: double, 2 CTAs)
#define FG_Q3_NXB 1
#endif
#ifndef FG_F32_Q2_COLLOC  // FP32 Q2 diffusion: collocated-gradient form (1) or packed sum factorisation (0)
#define FG_F32_Q2_COLLOC 1
#endif
#ifndef FG_F32_COLLOC_PACK  // FP32 collocated form: packed pairs in the interpolation passes (1) or scalar (0)
#define FG_F32_COLLOC_PACK 1
#endif
#ifndef FG_Q1_COLLOC  // Q1 diffusion (FP32 both formats, FP64 affine): collocated-gradient form (1) or not (0)
#define FG_Q1_COLLOC 1
#endif
#ifndef FG_F64_Q2A_COLLOC  // FP64 Q2 affine-format diffusion: collocated-gradient form (1) or sum factorisation (0)
#define FG_F64_Q2A_COLLOC 1
#endif
#ifndef FG_F32_Q3_COLLOC  // FP32 Q3 affine-format diffusion: collocated-gradient form (1) or sum factorisation (0)
#define FG_F32_Q3_COLLOC 1
#endif

namespace fg {

template <int OPK> struct NComp { static constexpr int v = OPK == 1 ? 1 : (OPK == 2 ? 6 : 7); };

// Quadrature-data layout: [item][warp][layer][col=(qy,qx)][qz][comp][lane].
template <int P, int OPK>
__host__ __device__ inline int64_t qd_index(const Grid &g, int item, int w, int lz, int col,
                                            int qz, int comp, int lane) {
    constexpr int Q = P + 1, NC = NComp<OPK>::v;
    return (((((int64_t)item * g.WY + w) * g.TZ + lz) * (Q * Q) + col) * Q + qz) * (NC * 32) +
           comp * 32 + lane;
}
template <int P, int OPK>
__host__ __device__ inline int64_t qd_size(const Grid &g) {
    constexpr int Q = P + 1, NC = NComp<OPK>::v;
    return (int64_t)g.n_items() * g.WY * g.TZ * Q * Q * Q * NC * 32;
}

template <typename T> struct ApplyArgs {
    Grid g;
    const T *qd;      // quadrature data (layout above)
    T *y;             // native-layout output
    T *face;          // per-item face slots (scratch)
    int accumulate;   // 1: y += A x, 0: y = A x
    int *err;         // device error word
    const int *skip;  // if non-null and *skip != 0 the kernel returns at once
    unsigned *fixcnt; // non-null: fix-up fused into the apply (per-item arrival counters, all zero
                      // between launches); null: fixup_kernel runs after the apply
    uint64_t wait_ns; // limit of each wait for a copy into shared memory; 0: 1 s
    int item0;        // first item of this launch (block b works on item item0 + b)
};

template <typename T, int P>
__device__ __forceinline__ void fused_fixup(const Grid &g, T *y, const T *face, unsigned *cnt,
                                            int item, int *flag);

// Quadrature-data formats.
//  FMT 0 (full): NC components per quadrature point (6 symmetric w|detJ| kappa
//    J^-1 J^-T, and/or w|detJ| rho); streamed one quadrature column per stage.
//  FMT 1 (affine-compressed, valid when J is constant over each element): per
//    element the 6 components of |detJ| J^-1 J^-T (diffusion), per quadrature
//    point the scalars w kappa c_k (diffusion) and/or w |detJ| rho c_m (mass);
//    streamed one element layer per stage.
//    layout [item][warp][layer][NCE + Q^3 NCQ][lane], NCE = 6 (diffusion) or 0,
//    quadrature point (col = qy*Q+qx, qz) at NCE + (col*Q + qz)*NCQ.
template <int OPK> struct AffineComp {
    static constexpr int NCE = (OPK & 2) ? 6 : 0;
    static constexpr int NCQ = ((OPK & 2) ? 1 : 0) + ((OPK & 1) ? 1 : 0);
};
template <int P, int OPK, int FMT> constexpr int stage_elems() {
    return FMT == 0 ? (P + 1) * NComp<OPK>::v * 32
                    : (AffineComp<OPK>::NCE + (P + 1) * (P + 1) * (P + 1) * AffineComp<OPK>::NCQ) * 32;
}
template <int P, int OPK, int FMT>
__host__ __device__ inline int64_t qd_size_fmt(const Grid &g) {
    // stages per layer: Q^2 columns (FMT 0) or 1 (FMT 1)
    constexpr int U = FMT == 0 ? (P + 1) * (P + 1) : 1;
    return (int64_t)g.n_items() * g.WY * g.TZ * U * stage_elems<P, OPK, FMT>();
}

// Shared-memory plan of the apply kernel (bytes).  NC here is the stage size
// in units of 32-lane vectors.
template <int P, typename T, int WY, int S, int NC> struct ApplySmem {
    static constexpr int D = P + 1, Q = P + 1;
    // x tile buffers: two (the next layer's tile loads during this layer's
    // math) except for Q3 in FP64, where one buffer lets 3 CTAs share an SM
    static constexpr int NXB = (P == 3 && sizeof(T) == 8) ? FG_Q3_NXB : 2;
    static constexpr int XW = round_up(32 * P + 1, 16 / (int)sizeof(T));
    static constexpr int RY = WY * P + 1;
    static constexpr int XTILE = (P + 1) * RY * XW;               // elements
    static constexpr int XB = round_up(XTILE * (int)sizeof(T), 128);
    static constexpr int STAGE = NC * 32;                         // elements
    static constexpr int QB = STAGE * (int)sizeof(T);
    static constexpr int off_q = NXB * XB;
    static constexpr int off_y = off_q + WY * S * QB;
    static constexpr int off_c = off_y + WY * D * D * 32 * (int)sizeof(T);
    static constexpr int off_b = round_up(off_c + D * D * WY * 32 * (int)sizeof(T), 8);
    static constexpr int bytes = off_b + (2 + WY * S) * 8;
};

// ---------------------------------------------------------------------------
// Merge of neighbouring element contributions and the scatter.  `out` holds
// the element result [c][b][a]; after this call every DOF of the item box is
// either stored into y (owned), or into the face slot of the item (owned by a
// neighbour item).  `essval(c,b,a)` returns the value written on essential
// DOFs (x for the constrained apply, 1 for the diagonal).
// ---------------------------------------------------------------------------
template <int P, typename T, int WY, class EssVal>
__device__ __forceinline__ void merge_and_store(T (&out)[P + 1][P + 1][P + 1], const Grid &g,
                                                T *ybuf, T *carry, int lz, int nl, int tz,
                                                int warp, int lane, int item, bool valid,
                                                int lane_last, int w_last, bool fx0, bool fx1,
                                                bool fy0, bool fy1, bool fz0, bool fz1, T *y,
                                                T *face, int accumulate, EssVal essval) {
    constexpr int D = P + 1;
    constexpr int NT = WY * 32;
    // x: lane l receives the a=P face of lane l-1 into its a=0 face
#pragma unroll
    for (int c = 0; c < D; ++c)
#pragma unroll
        for (int b = 0; b < D; ++b) {
            T v = __shfl_up_sync(0xffffffffu, out[c][b][P], 1);
            if (lane > 0) out[c][b][0] += v;
        }
    // y: row warp w receives the b=P row of warp w-1 into its b=0 row
    T *yb = ybuf + warp * (D * D * 32);
#pragma unroll
    for (int c = 0; c < D; ++c)
#pragma unroll
        for (int a = 0; a < D; ++a) yb[(c * D + a) * 32 + lane] = out[c][P][a];
    __syncthreads();
    if (warp > 0) {
        const T *yp = ybuf + (warp - 1) * (D * D * 32);
#pragma unroll
        for (int c = 0; c < D; ++c)
#pragma unroll
            for (int a = 0; a < D; ++a) out[c][0][a] += yp[(c * D + a) * 32 + lane];
    }
    // z: layer lz receives the c=P plane of layer lz-1 into its c=0 plane
    const int tid = warp * 32 + lane;
    if (lz > 0) {
#pragma unroll
        for (int b = 0; b < D; ++b)
#pragma unroll
            for (int a = 0; a < D; ++a) out[0][b][a] += carry[(b * D + a) * NT + tid];
    }
    if (lz + 1 < nl) {
#pragma unroll
        for (int b = 0; b < D; ++b)
#pragma unroll
            for (int a = 0; a < D; ++a) carry[(b * D + a) * NT + tid] = out[P][b][a];
    }
    if (!valid) return;
    const int tx = item % g.ntx, ty = (item / g.ntx) % g.nty;
    const int I0 = tx * 32 * P, J0 = ty * WY * P, K0 = tz * g.TZ * P;
    const int ex = tx * 32 + lane, ey = ty * WY + warp, ez = tz * g.TZ + lz;
    const int SX = 32 * P + 1, SY = WY * P + 1;
    T *fxp = face + (int64_t)item * g.face_stride();
    T *fyp = fxp + g.fx();
    T *fzp = fyp + g.fy();
    const bool last_layer = (lz == nl - 1);
#pragma unroll
    for (int c = 0; c < D; ++c) {
        if (c == P && !last_layer) continue;
        const int K = K0 + P * lz + c;
        const bool zhi = (c == P) && (ez != g.nz - 1);
#pragma unroll
        for (int b = 0; b < D; ++b) {
            if (b == P && warp != w_last) continue;
            const int J = J0 + P * warp + b;
            const bool yhi = (b == P) && (ey != g.ny - 1);
#pragma unroll
            for (int a = 0; a < D; ++a) {
                if (a == P && lane != lane_last) continue;
                const int I = I0 + P * lane + a;
                const bool xhi = (a == P) && (ex != g.nx - 1);
                T v = out[c][b][a];
                if (xhi) {
                    fxp[(K - K0) * SY + (J - J0)] = v;
                } else if (yhi) {
                    fyp[(K - K0) * SX + (I - I0)] = v;
                } else if (zhi) {
                    fzp[(J - J0) * SX + (I - I0)] = v;
                } else {
                    const bool e = (a == 0 && fx0) || (a == P && fx1) || (b == 0 && fy0) ||
                                   (b == P && fy1) || (c == 0 && fz0) || (c == P && fz1);
                    if (e) v = essval(c, b, a);
                    const int64_t d = g.dof(I, J, K);
                    y[d] = accumulate ? y[d] + v : v;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// The apply kernel.
// ---------------------------------------------------------------------------
template <int P, int OPK, typename T, int WY, int S, int FMT>
__device__ __forceinline__ void pa_apply_body(const CUtensorMap *xmap_ptr, const ApplyArgs<T> &A,
                                              const int item) {
    constexpr int D = P + 1, Q = P + 1, NC = NComp<OPK>::v;
    constexpr bool HM = (OPK & 1) != 0, HK = (OPK & 2) != 0;
    constexpr int COLS = Q * Q;
    constexpr int UPL = FMT == 0 ? COLS : 1;  // stream units per layer
    constexpr int NCE = AffineComp<OPK>::NCE, NCQ = AffineComp<OPK>::NCQ;
    using SM = ApplySmem<P, T, WY, S, stage_elems<P, OPK, FMT>() / 32>;
    constexpr int STAGE = SM::STAGE, XW = SM::XW, RY = SM::RY;
    using TB = Tab<T>;

    if (A.skip && *A.skip) return;
    const Grid g = A.g;
    const uint64_t wlim = A.wait_ns ? A.wait_ns : 1000000000ull;
    const CUtensorMap &xmap = *xmap_ptr;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T *xs = reinterpret_cast<T *>(smem_raw);
    T *qs = reinterpret_cast<T *>(smem_raw + SM::off_q);
    T *ybuf = reinterpret_cast<T *>(smem_raw + SM::off_y);
    T *carry = reinterpret_cast<T *>(smem_raw + SM::off_c);
    uint64_t *xbar = reinterpret_cast<uint64_t *>(smem_raw + SM::off_b);
    uint64_t *qbar = xbar + 2;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tx = item % g.ntx, ty = (item / g.ntx) % g.nty, tz = item / (g.ntx * g.nty);
    const int nl = min(g.TZ, g.nz - tz * g.TZ);
    const int ex = tx * 32 + lane, ey = ty * WY + warp;
    const bool valid = ex < g.nx && ey < g.ny;
    const int lane_last = min(31, g.nx - 1 - tx * 32);
    const int w_last = min(WY - 1, g.ny - 1 - ty * WY);
    const int I0 = tx * 32 * P, J0 = ty * WY * P, K0 = tz * g.TZ * P;
    const int total_cols = nl * UPL;
    const T *qdw = A.qd + (int64_t)(item * WY + warp) * g.TZ * UPL * STAGE;
    T *qsw = qs + warp * S * STAGE;
    uint64_t *qbw = qbar + warp * S;
    constexpr uint32_t XBYTES = (uint32_t)(SM::XTILE * sizeof(T));
    constexpr uint32_t QBYTES = (uint32_t)SM::QB;

    if (threadIdx.x == 0) {
        prefetch_tmap(&xmap);
        mbar_init(&xbar[0], 1);
        mbar_init(&xbar[1], 1);
        for (int i = 0; i < WY * S; ++i) mbar_init(&qbar[i], 1);
        fence_barrier_init();
    }
    __syncthreads();
    int x_issued = 0, q_issued = 0;  // thread 0 / lane 0 bookkeeping
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(&xbar[0], XBYTES);
        tma_load_3d(xs, &xmap, I0, J0, K0, &xbar[0]);
        x_issued = 1;
    }
    if (lane == 0) {
        for (int j = 0; j < S && j < total_cols; ++j) {
            mbar_arrive_expect_tx(&qbw[j], QBYTES);
            bulk_g2s(qsw + j * STAGE, qdw + (int64_t)j * STAGE, QBYTES, &qbw[j]);
            q_issued = j + 1;
        }
    }
    const int ess = g.ess;
    const bool fx0 = (ess & 16) && ex == 0, fx1 = (ess & 32) && ex == g.nx - 1;
    const bool fy0 = (ess & 4) && ey == 0, fy1 = (ess & 8) && ey == g.ny - 1;
    bool ok = true;
    int x_waited = 0, q_waited = 0;

    for (int lz = 0; lz < nl; ++lz) {
        const int ez = tz * g.TZ + lz;
        const bool fz0 = (ess & 1) && ez == 0, fz1 = (ess & 2) && ez == g.nz - 1;
        constexpr int NXB = SM::NXB;
        const int xb = lz % NXB;
        if (threadIdx.x == 0 && ok && (NXB == 2 ? lz + 1 < nl : lz > 0)) {
            // double buffer: buffer (lz+1)&1 was last read in layer lz-1, before the
            // end-of-layer barrier; single buffer: layer lz loads now, after that barrier
            const int ln = NXB == 2 ? lz + 1 : lz, bn = ln % NXB;
            fence_proxy_async();
            mbar_arrive_expect_tx(&xbar[bn], XBYTES);
            tma_load_3d(reinterpret_cast<unsigned char *>(xs) + bn * SM::XB, &xmap, I0, J0, K0 + ln * P,
                        &xbar[bn]);
            x_issued = ln + 1;
        }
        wait_stage(&xbar[xb], (lz / NXB) & 1, A.err, wlim, ok, x_waited, lz + 1);
        const T *xt = reinterpret_cast<const T *>(reinterpret_cast<const unsigned char *>(xs) +
                                                  xb * SM::XB);

        T out[D][D][D];
        if constexpr (HK && ((std::is_same<T, float>::value &&
                               ((P == 1 && FG_Q1_COLLOC) || (P == 2 && FG_F32_Q2_COLLOC) ||
                                (P == 3 && FMT == 1 && FG_F32_Q3_COLLOC))) ||
                              (std::is_same<T, double>::value && FMT == 1 &&
                               ((P == 1 && FG_Q1_COLLOC) || (P == 2 && FG_F64_Q2A_COLLOC))))) {
            // FP32 Q2 / Q3-affine and FP64 Q2-affine diffusion (+ mass), collocated form: the element values are
            // interpolated to the Gauss points (uq = (B x B x B) u), the gradient
            // at a point is the collocated derivative Dq = G B^-1 along the
            // point's three lines of uq, D is applied per point, the transposed
            // derivatives accumulate into a point field w, and the result is
            // (B^T x B^T x B^T) w.  The same operator as the sum factorisation
            // with B and G (G = Dq B): Q2 1296 instead of 1620 FMAs an element and
            // 54 live values instead of 81; Q3 3648 instead of ~5700 FMAs with 128
            // live values (faster than the slab form on the affine format, slower
            // on the full format, where the slab form's smaller state wins).
            using TBf = Tab<T>;
            T uq[Q][Q][Q];  // [qz][qy][qx]
            if constexpr (std::is_same<T, float>::value && FG_F32_COLLOC_PACK) {
                // x and y passes as packed pairs of DOF planes (c, c+1), loaded
                // straight into register pairs; the z pass reads the halves in
                // plane order.  Every lane does the scalar code's FMA in its
                // order, so the result is the same bit for bit.
                constexpr int NPC = D / 2;
                float2 up[NPC][D][D];
                float us[D][D];
                auto ld = [&](int c, int b, int a) -> float {
                    const float v = xt[(c * RY + warp * P + b) * XW + lane * P + a];
                    const bool e = (a == 0 && fx0) || (a == P && fx1) || (b == 0 && fy0) || (b == P && fy1) ||
                                   (c == 0 && fz0) || (c == P && fz1);
                    return e ? 0.f : v;
                };
#pragma unroll
                for (int b = 0; b < D; ++b)
#pragma unroll
                    for (int a = 0; a < D; ++a) {
#pragma unroll
                        for (int cp = 0; cp < NPC; ++cp) up[cp][b][a] = make_float2(ld(2 * cp, b, a), ld(2 * cp + 1, b, a));
                        if (D & 1) us[b][a] = ld(D - 1, b, a);
                    }
                float2 t1p[NPC][D][Q];
                float t1s[D][Q];
#pragma unroll
                for (int b = 0; b < D; ++b)
#pragma unroll
                    for (int qx = 0; qx < Q; ++qx) {
#pragma unroll
                        for (int cp = 0; cp < NPC; ++cp) {
                            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                            for (int a = 0; a < D; ++a) acc = __ffma2_rn(c_BB32[P - 1][qx][a], up[cp][b][a], acc);
                            t1p[cp][b][qx] = acc;
                        }
                        if (D & 1) {
                            float s0 = 0.f;
#pragma unroll
                            for (int a = 0; a < D; ++a) s0 += TBf::B(P, qx, a) * us[b][a];
                            t1s[b][qx] = s0;
                        }
                    }
                float2 t2p[NPC][Q][Q];
                float t2s[Q][Q];
#pragma unroll
                for (int qy = 0; qy < Q; ++qy)
#pragma unroll
                    for (int qx = 0; qx < Q; ++qx) {
#pragma unroll
                        for (int cp = 0; cp < NPC; ++cp) {
                            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                            for (int b = 0; b < D; ++b) acc = __ffma2_rn(c_BB32[P - 1][qy][b], t1p[cp][b][qx], acc);
                            t2p[cp][qy][qx] = acc;
                        }
                        if (D & 1) {
                            float s0 = 0.f;
#pragma unroll
                            for (int b = 0; b < D; ++b) s0 += TBf::B(P, qy, b) * t1s[b][qx];
                            t2s[qy][qx] = s0;
                        }
                    }
#pragma unroll
                for (int qz = 0; qz < Q; ++qz)
#pragma unroll
                    for (int qy = 0; qy < Q; ++qy)
#pragma unroll
                        for (int qx = 0; qx < Q; ++qx) {
                            float s0 = 0.f;
#pragma unroll
                            for (int cp = 0; cp < NPC; ++cp) {
                                s0 += TBf::B(P, qz, 2 * cp) * t2p[cp][qy][qx].x;
                                s0 += TBf::B(P, qz, 2 * cp + 1) * t2p[cp][qy][qx].y;
                            }
                            if (D & 1) s0 += TBf::B(P, qz, D - 1) * t2s[qy][qx];
                            uq[qz][qy][qx] = s0;
                        }
            } else {
                T u[D][D][D];
#pragma unroll
                for (int c = 0; c < D; ++c)
#pragma unroll
                    for (int b = 0; b < D; ++b)
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            const T v = xt[(c * RY + warp * P + b) * XW + lane * P + a];
                            const bool e = (a == 0 && fx0) || (a == P && fx1) || (b == 0 && fy0) ||
                                           (b == P && fy1) || (c == 0 && fz0) || (c == P && fz1);
                            u[c][b][a] = e ? T(0) : v;
                        }
                T t1[D][D][Q];  // [c][b][qx]
#pragma unroll
                for (int c = 0; c < D; ++c)
#pragma unroll
                    for (int b = 0; b < D; ++b)
#pragma unroll
                        for (int qx = 0; qx < Q; ++qx) {
                            T s0 = T(0);
#pragma unroll
                            for (int a = 0; a < D; ++a) s0 += TBf::B(P, qx, a) * u[c][b][a];
                            t1[c][b][qx] = s0;
                        }
                T t2[D][Q][Q];  // [c][qy][qx]
#pragma unroll
                for (int c = 0; c < D; ++c)
#pragma unroll
                    for (int qy = 0; qy < Q; ++qy)
#pragma unroll
                        for (int qx = 0; qx < Q; ++qx) {
                            T s0 = T(0);
#pragma unroll
                            for (int b = 0; b < D; ++b) s0 += TBf::B(P, qy, b) * t1[c][b][qx];
                            t2[c][qy][qx] = s0;
                        }
#pragma unroll
                for (int qz = 0; qz < Q; ++qz)
#pragma unroll
                    for (int qy = 0; qy < Q; ++qy)
#pragma unroll
                        for (int qx = 0; qx < Q; ++qx) {
                            T s0 = T(0);
#pragma unroll
                            for (int c = 0; c < D; ++c) s0 += TBf::B(P, qz, c) * t2[c][qy][qx];
                            uq[qz][qy][qx] = s0;
                        }
            }
            // point field w: FP32 as pairs of adjacent qx (wp) and the last qx of an
            // odd Q (ws), so the transposed z and y passes run packed; FP64 plain
            constexpr int NPX = Q / 2;
            T w[Q][Q][Q];
            float2 wp[Q][Q][NPX > 0 ? NPX : 1];
            float ws[Q][Q];
            auto W = [&](int qz, int qy, int qx) -> T & {
                if constexpr (std::is_same<T, float>::value && FG_F32_COLLOC_PACK) {
                    if (qx < 2 * NPX) return (qx & 1) ? wp[qz][qy][qx >> 1].y : wp[qz][qy][qx >> 1].x;
                    return ws[qz][qy];
                } else {
                    return w[qz][qy][qx];
                }
            };
#pragma unroll
            for (int qz = 0; qz < Q; ++qz)
#pragma unroll
                for (int qy = 0; qy < Q; ++qy)
#pragma unroll
                    for (int qx = 0; qx < Q; ++qx) W(qz, qy, qx) = T(0);
            T Ge[6] = {0, 0, 0, 0, 0, 0};
            const T *ql = nullptr;
            if (FMT == 1) {
                const int j = lz, s = j % S;
                wait_stage(&qbw[s], (j / S) & 1, A.err, wlim, ok, q_waited, j + 1);
                ql = qsw + s * STAGE;
#pragma unroll
                for (int k = 0; k < NCE; ++k) Ge[k] = ql[k * 32 + lane];
            }
#pragma unroll
            for (int qy = 0; qy < Q; ++qy)
#pragma unroll
                for (int qx = 0; qx < Q; ++qx) {
                    const int col = qy * Q + qx;
                    const int j = lz * COLS + col;
                    const int s = j % S;
                    if (FMT == 0) wait_stage(&qbw[s], (j / S) & 1, A.err, wlim, ok, q_waited, j + 1);
                    const T *qc = FMT == 0 ? qsw + s * STAGE : ql;
#pragma unroll
                    for (int qz = 0; qz < Q; ++qz) {
                        T gx = T(0), gy = T(0), gz = T(0);
#pragma unroll
                        for (int k = 0; k < Q; ++k) {
                            gx += TBf::DQ(P, qx, k) * uq[qz][qy][k];
                            gy += TBf::DQ(P, qy, k) * uq[qz][k][qx];
                            gz += TBf::DQ(P, qz, k) * uq[k][qy][qx];
                        }
                        T vx, vy, vz, vu = T(0);
                        if (FMT == 0) {
                            const T *qq = qc + qz * (NC * 32) + lane;
                            const T d0 = qq[0], d1 = qq[32], d2 = qq[64], d3 = qq[96], d4 = qq[128], d5 = qq[160];
                            vx = d0 * gx + d1 * gy + d2 * gz;
                            vy = d1 * gx + d3 * gy + d4 * gz;
                            vz = d2 * gx + d4 * gy + d5 * gz;
                            if (HM) vu = qq[6 * 32] * uq[qz][qy][qx];
                        } else {
                            const T *qq = qc + (NCE + (col * Q + qz) * NCQ) * 32 + lane;
                            const T sk = qq[0];
                            const T hx = sk * gx, hy = sk * gy, hz = sk * gz;
                            vx = Ge[0] * hx + Ge[1] * hy + Ge[2] * hz;
                            vy = Ge[1] * hx + Ge[3] * hy + Ge[4] * hz;
                            vz = Ge[2] * hx + Ge[4] * hy + Ge[5] * hz;
                            if (HM) vu = qq[32] * uq[qz][qy][qx];
                        }
#pragma unroll
                        for (int k = 0; k < Q; ++k) {
                            W(qz, qy, k) += TBf::DQ(P, qx, k) * vx;
                            W(qz, k, qx) += TBf::DQ(P, qy, k) * vy;
                            W(k, qy, qx) += TBf::DQ(P, qz, k) * vz;
                        }
                        if (HM) W(qz, qy, qx) += vu;
                    }
                    if (FMT == 0) {
                        __syncwarp();
                        if (lane == 0 && ok && j + S < total_cols) {
                            fence_proxy_async();
                            mbar_arrive_expect_tx(&qbw[s], QBYTES);
                            bulk_g2s(qsw + s * STAGE, qdw + (int64_t)(j + S) * STAGE, QBYTES, &qbw[s]);
                            q_issued = j + S + 1;
                        }
                    }
                }
            if (FMT == 1) {
                const int j = lz, s = j % S;
                __syncwarp();
                if (lane == 0 && ok && j + S < total_cols) {
                    fence_proxy_async();
                    mbar_arrive_expect_tx(&qbw[s], QBYTES);
                    bulk_g2s(qsw + s * STAGE, qdw + (int64_t)(j + S) * STAGE, QBYTES, &qbw[s]);
                    q_issued = j + S + 1;
                }
            }
            if constexpr (std::is_same<T, float>::value && FG_F32_COLLOC_PACK) {
                // transposed z and y passes packed over pairs of qx, then x from the halves
                float2 s1p[D][Q][NPX > 0 ? NPX : 1];
                float s1s[D][Q];
#pragma unroll
                for (int c = 0; c < D; ++c)
#pragma unroll
                    for (int qy = 0; qy < Q; ++qy) {
#pragma unroll
                        for (int xp = 0; xp < NPX; ++xp) {
                            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                            for (int qz = 0; qz < Q; ++qz) acc = __ffma2_rn(c_BB32[P - 1][qz][c], wp[qz][qy][xp], acc);
                            s1p[c][qy][xp] = acc;
                        }
                        if (Q & 1) {
                            float t = 0.f;
#pragma unroll
                            for (int qz = 0; qz < Q; ++qz) t += TBf::B(P, qz, c) * ws[qz][qy];
                            s1s[c][qy] = t;
                        }
                    }
                float2 s2p[D][D][NPX > 0 ? NPX : 1];
                float s2s[D][D];
#pragma unroll
                for (int c = 0; c < D; ++c)
#pragma unroll
                    for (int b = 0; b < D; ++b) {
#pragma unroll
                        for (int xp = 0; xp < NPX; ++xp) {
                            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                            for (int qy = 0; qy < Q; ++qy) acc = __ffma2_rn(c_BB32[P - 1][qy][b], s1p[c][qy][xp], acc);
                            s2p[c][b][xp] = acc;
                        }
                        if (Q & 1) {
                            float t = 0.f;
#pragma unroll
                            for (int qy = 0; qy < Q; ++qy) t += TBf::B(P, qy, b) * s1s[c][qy];
                            s2s[c][b] = t;
                        }
                    }
#pragma unroll
                for (int c = 0; c < D; ++c)
#pragma unroll
                    for (int b = 0; b < D; ++b)
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            float t = 0.f;
#pragma unroll
                            for (int xp = 0; xp < NPX; ++xp) {
                                t += TBf::B(P, 2 * xp, a) * s2p[c][b][xp].x;
                                t += TBf::B(P, 2 * xp + 1, a) * s2p[c][b][xp].y;
                            }
                            if (Q & 1) t += TBf::B(P, Q - 1, a) * s2s[c][b];
                            out[c][b][a] = t;
                        }
            } else {
                T s1[D][Q][Q];  // [c][qy][qx]
#pragma unroll
                for (int c = 0; c < D; ++c)
#pragma unroll
                    for (int qy = 0; qy < Q; ++qy)
#pragma unroll
                        for (int qx = 0; qx < Q; ++qx) {
                            T t = T(0);
#pragma unroll
                            for (int qz = 0; qz < Q; ++qz) t += TBf::B(P, qz, c) * w[qz][qy][qx];
                            s1[c][qy][qx] = t;
                        }
                T s2[D][D][Q];  // [c][b][qx]
#pragma unroll
                for (int c = 0; c < D; ++c)
#pragma unroll
                    for (int b = 0; b < D; ++b)
#pragma unroll
                        for (int qx = 0; qx < Q; ++qx) {
                            T t = T(0);
#pragma unroll
                            for (int qy = 0; qy < Q; ++qy) t += TBf::B(P, qy, b) * s1[c][qy][qx];
                            s2[c][b][qx] = t;
                        }
#pragma unroll
                for (int c = 0; c < D; ++c)
#pragma unroll
                    for (int b = 0; b < D; ++b)
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            T t = T(0);
#pragma unroll
                            for (int qx = 0; qx < Q; ++qx) t += TBf::B(P, qx, a) * s2[c][b][qx];
                            out[c][b][a] = t;
                        }
            }
        } else if constexpr (std::is_same<T, float>::value && P == 2 && HK) {
            // FP32 Q2 diffusion (+ mass): the contractions as packed pairs, two
            // FP32 FMAs per instruction (__ffma2_rn).  Pairing: x gives
            // (A1, A0) = (Gx, Bx)(u, u); y gives (C2, C1) = (By, Gy)(A1, A0) and
            // C0 = By A0; z gives (gx, gy) = (Bz, Bz)(C2, C1), gz = Gz C0; the
            // transposed passes pair the same way.  Per element 486 paired and
            // 567 single FMAs instead of 1539 single ones.
            float u[D][D][D];
#pragma unroll
            for (int c = 0; c < D; ++c)
#pragma unroll
                for (int b = 0; b < D; ++b)
#pragma unroll
                    for (int a = 0; a < D; ++a) {
                        const float v = xt[(c * RY + warp * P + b) * XW + lane * P + a];
                        const bool e = (a == 0 && fx0) || (a == P && fx1) || (b == 0 && fy0) ||
                                       (b == P && fy1) || (c == 0 && fz0) || (c == P && fz1);
                        u[c][b][a] = e ? 0.f : v;
                    }
            float2 C21[D][Q][Q];  // (C2, C1) [c][qy][qx]
            float C0[D][Q][Q];
#pragma unroll
            for (int c = 0; c < D; ++c) {
                float2 X[D][Q];  // (A1, A0) [b][qx]
#pragma unroll
                for (int b = 0; b < D; ++b)
#pragma unroll
                    for (int qx = 0; qx < Q; ++qx) {
                        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                        for (int a = 0; a < D; ++a)
                            acc = __ffma2_rn(c_GB32[P - 1][qx][a], make_float2(u[c][b][a], u[c][b][a]), acc);
                        X[b][qx] = acc;
                    }
#pragma unroll
                for (int qy = 0; qy < Q; ++qy)
#pragma unroll
                    for (int qx = 0; qx < Q; ++qx) {
                        float2 acc = make_float2(0.f, 0.f);
                        float c0 = 0.f;
#pragma unroll
                        for (int b = 0; b < D; ++b) {
                            acc = __ffma2_rn(c_BG32[P - 1][qy][b], X[b][qx], acc);
                            c0 += TB::B(P, qy, b) * X[b][qx].y;
                        }
                        C21[c][qy][qx] = acc;
                        C0[c][qy][qx] = c0;
                    }
            }
            T Ge[6] = {0, 0, 0, 0, 0, 0};
            const T *ql = nullptr;
            if (FMT == 1) {
                const int j = lz;
                const int s = j % S;
                wait_stage(&qbw[s], (j / S) & 1, A.err, wlim, ok, q_waited, j + 1);
                ql = qsw + s * STAGE;
#pragma unroll
                for (int k = 0; k < NCE; ++k) Ge[k] = ql[k * 32 + lane];
            }
#pragma unroll
            for (int qy = 0; qy < Q; ++qy)
#pragma unroll
                for (int qx = 0; qx < Q; ++qx) {
                    const int col = qy * Q + qx;
                    const int j = lz * COLS + col;
                    const int s = j % S;
                    if (FMT == 0) {
                        wait_stage(&qbw[s], (j / S) & 1, A.err, wlim, ok, q_waited, j + 1);
                    }
                    const T *qc = FMT == 0 ? qsw + s * STAGE : ql;
                    float2 vxy[Q];
                    float vz[Q], vu[Q];
#pragma unroll
                    for (int qz = 0; qz < Q; ++qz) {
                        float2 g21 = make_float2(0.f, 0.f);
                        float gz = 0.f, ui = 0.f;
#pragma unroll
                        for (int c = 0; c < D; ++c) {
                            g21 = __ffma2_rn(c_BB32[P - 1][qz][c], C21[c][qy][qx], g21);
                            gz += TB::G(P, qz, c) * C0[c][qy][qx];
                            if (HM) ui += TB::B(P, qz, c) * C0[c][qy][qx];
                        }
                        const float gx = g21.x, gy = g21.y;
                        float vx, vy;
                        if (FMT == 0) {
                            const T *qq = qc + qz * (NC * 32) + lane;
                            const T d0 = qq[0], d1 = qq[32], d2 = qq[64], d3 = qq[96], d4 = qq[128], d5 = qq[160];
                            vx = d0 * gx + d1 * gy + d2 * gz;
                            vy = d1 * gx + d3 * gy + d4 * gz;
                            vz[qz] = d2 * gx + d4 * gy + d5 * gz;
                            vu[qz] = HM ? qq[6 * 32] * ui : 0.f;
                        } else {
                            const T *qq = qc + (NCE + (col * Q + qz) * NCQ) * 32 + lane;
                            const T sk = qq[0];
                            const T hx = sk * gx, hy = sk * gy, hz = sk * gz;
                            vx = Ge[0] * hx + Ge[1] * hy + Ge[2] * hz;
                            vy = Ge[1] * hx + Ge[3] * hy + Ge[4] * hz;
                            vz[qz] = Ge[2] * hx + Ge[4] * hy + Ge[5] * hz;
                            vu[qz] = HM ? qq[32] * ui : 0.f;
                        }
                        vxy[qz] = make_float2(vx, vy);
                    }
#pragma unroll
                    for (int c = 0; c < D; ++c) {
                        float2 e21 = make_float2(0.f, 0.f);
                        float e0 = 0.f;
#pragma unroll
                        for (int qz = 0; qz < Q; ++qz) {
                            e21 = __ffma2_rn(c_BB32[P - 1][qz][c], vxy[qz], e21);
                            e0 += TB::G(P, qz, c) * vz[qz];
                            if (HM) e0 += TB::B(P, qz, c) * vu[qz];
                        }
                        C21[c][qy][qx] = e21;
                        C0[c][qy][qx] = e0;
                    }
                    if (FMT == 0) {
                        __syncwarp();
                        if (lane == 0 && ok && j + S < total_cols) {
                            fence_proxy_async();
                            mbar_arrive_expect_tx(&qbw[s], QBYTES);
                            bulk_g2s(qsw + s * STAGE, qdw + (int64_t)(j + S) * STAGE, QBYTES, &qbw[s]);
                            q_issued = j + S + 1;
                        }
                    }
                }
            if (FMT == 1) {
                const int j = lz, s = j % S;
                __syncwarp();
                if (lane == 0 && ok && j + S < total_cols) {
                    fence_proxy_async();
                    mbar_arrive_expect_tx(&qbw[s], QBYTES);
                    bulk_g2s(qsw + s * STAGE, qdw + (int64_t)(j + S) * STAGE, QBYTES, &qbw[s]);
                    q_issued = j + S + 1;
                }
            }
#pragma unroll
            for (int c = 0; c < D; ++c) {
                float2 F[D][Q];  // (F1, F0) [b][qx]
#pragma unroll
                for (int b = 0; b < D; ++b)
#pragma unroll
                    for (int qx = 0; qx < Q; ++qx) {
                        float2 acc = make_float2(0.f, 0.f);
                        float f0 = 0.f;
#pragma unroll
                        for (int qy = 0; qy < Q; ++qy) {
                            acc = __ffma2_rn(c_BG32[P - 1][qy][b], C21[c][qy][qx], acc);
                            f0 += TB::B(P, qy, b) * C0[c][qy][qx];
                        }
                        F[b][qx] = make_float2(acc.x, acc.y + f0);
                    }
#pragma unroll
                for (int b = 0; b < D; ++b)
#pragma unroll
                    for (int a = 0; a < D; ++a) {
                        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                        for (int qx = 0; qx < Q; ++qx) acc = __ffma2_rn(c_GB32[P - 1][qx][a], F[b][qx], acc);
                        out[c][b][a] = acc.x + acc.y;
                    }
            }
        } else if constexpr (P != 3 || (FMT == 1 && sizeof(T) == 4)) {
            // ---- gather (E) with essential-DOF masking -------------------------
            T u[D][D][D];
    #pragma unroll
            for (int c = 0; c < D; ++c)
    #pragma unroll
                for (int b = 0; b < D; ++b)
    #pragma unroll
                    for (int a = 0; a < D; ++a) {
                        const T v = xt[(c * RY + warp * P + b) * XW + lane * P + a];
                        const bool e = (a == 0 && fx0) || (a == P && fx1) || (b == 0 && fy0) ||
                                       (b == P && fy1) || (c == 0 && fz0) || (c == P && fz1);
                        u[c][b][a] = e ? T(0) : v;
                    }
            // ---- B: contractions in x then y ----------------------------------
            T C0[D][Q][Q], C1[D][Q][Q], C2[D][Q][Q];  // [c][qy][qx]
    #pragma unroll
            for (int c = 0; c < D; ++c) {
                T A0[D][Q], A1[D][Q];
    #pragma unroll
                for (int b = 0; b < D; ++b)
    #pragma unroll
                    for (int qx = 0; qx < Q; ++qx) {
                        T s0 = 0, s1 = 0;
    #pragma unroll
                        for (int a = 0; a < D; ++a) {
                            s0 += TB::B(P, qx, a) * u[c][b][a];
                            if (HK) s1 += TB::G(P, qx, a) * u[c][b][a];
                        }
                        A0[b][qx] = s0;
                        A1[b][qx] = s1;
                    }
    #pragma unroll
                for (int qy = 0; qy < Q; ++qy)
    #pragma unroll
                    for (int qx = 0; qx < Q; ++qx) {
                        T s0 = 0, s1 = 0, s2 = 0;
    #pragma unroll
                        for (int b = 0; b < D; ++b) {
                            s0 += TB::B(P, qy, b) * A0[b][qx];
                            if (HK) {
                                s1 += TB::G(P, qy, b) * A0[b][qx];
                                s2 += TB::B(P, qy, b) * A1[b][qx];
                            }
                        }
                        C0[c][qy][qx] = s0;
                        C1[c][qy][qx] = s1;
                        C2[c][qy][qx] = s2;
                    }
            }
            // ---- per quadrature column: B in z, D, B^T in z (in place) --------
            T Ge[6] = {0, 0, 0, 0, 0, 0};
            const T *ql = nullptr;  // layer stage (FMT 1)
            if (FMT == 1) {
                const int j = lz;
                const int s = j % S;
                wait_stage(&qbw[s], (j / S) & 1, A.err, wlim, ok, q_waited, j + 1);
                ql = qsw + s * STAGE;
    #pragma unroll
                for (int k = 0; k < NCE; ++k) Ge[k] = ql[k * 32 + lane];
            }
    #pragma unroll
            for (int qy = 0; qy < Q; ++qy)
    #pragma unroll
                for (int qx = 0; qx < Q; ++qx) {
                    const int col = qy * Q + qx;
                    const int j = lz * COLS + col;
                    const int s = j % S;
                    if (FMT == 0) {
                        wait_stage(&qbw[s], (j / S) & 1, A.err, wlim, ok, q_waited, j + 1);
                    }
                    const T *qc = FMT == 0 ? qsw + s * STAGE : ql;
                    T vx[Q], vy[Q], vz[Q], vu[Q];
    #pragma unroll
                    for (int qz = 0; qz < Q; ++qz) {
                        T gx = 0, gy = 0, gz = 0, ui = 0;
    #pragma unroll
                        for (int c = 0; c < D; ++c) {
                            if (HK) {
                                gx += TB::B(P, qz, c) * C2[c][qy][qx];
                                gy += TB::B(P, qz, c) * C1[c][qy][qx];
                                gz += TB::G(P, qz, c) * C0[c][qy][qx];
                            }
                            if (HM) ui += TB::B(P, qz, c) * C0[c][qy][qx];
                        }
                        if (FMT == 0) {
                            const T *qq = qc + qz * (NC * 32) + lane;
                            if (HK) {
                                const T d0 = qq[0], d1 = qq[32], d2 = qq[64], d3 = qq[96], d4 = qq[128],
                                        d5 = qq[160];
                                vx[qz] = d0 * gx + d1 * gy + d2 * gz;
                                vy[qz] = d1 * gx + d3 * gy + d4 * gz;
                                vz[qz] = d2 * gx + d4 * gy + d5 * gz;
                            }
                            if (HM) vu[qz] = qq[(HK ? 6 : 0) * 32] * ui;
                        } else {
                            const T *qq = qc + (NCE + (col * Q + qz) * NCQ) * 32 + lane;
                            if (HK) {
                                const T sk = qq[0];
                                const T hx = sk * gx, hy = sk * gy, hz = sk * gz;
                                vx[qz] = Ge[0] * hx + Ge[1] * hy + Ge[2] * hz;
                                vy[qz] = Ge[1] * hx + Ge[3] * hy + Ge[4] * hz;
                                vz[qz] = Ge[2] * hx + Ge[4] * hy + Ge[5] * hz;
                            }
                            if (HM) vu[qz] = qq[(HK ? 1 : 0) * 32] * ui;
                        }
                    }
    #pragma unroll
                    for (int c = 0; c < D; ++c) {
                        T e0 = 0, e1 = 0, e2 = 0;
    #pragma unroll
                        for (int qz = 0; qz < Q; ++qz) {
                            if (HK) {
                                e2 += TB::B(P, qz, c) * vx[qz];
                                e1 += TB::B(P, qz, c) * vy[qz];
                                e0 += TB::G(P, qz, c) * vz[qz];
                            }
                            if (HM) e0 += TB::B(P, qz, c) * vu[qz];
                        }
                        C0[c][qy][qx] = e0;
                        C1[c][qy][qx] = e1;
                        C2[c][qy][qx] = e2;
                    }
                    if (FMT == 0) {
                        __syncwarp();
                        if (lane == 0 && ok && j + S < total_cols) {
                            fence_proxy_async();
                            mbar_arrive_expect_tx(&qbw[s], QBYTES);
                            bulk_g2s(qsw + s * STAGE, qdw + (int64_t)(j + S) * STAGE, QBYTES, &qbw[s]);
                            q_issued = j + S + 1;
                        }
                    }
                }
            if (FMT == 1) {
                const int j = lz, s = j % S;
                __syncwarp();
                if (lane == 0 && ok && j + S < total_cols) {
                    fence_proxy_async();
                    mbar_arrive_expect_tx(&qbw[s], QBYTES);
                    bulk_g2s(qsw + s * STAGE, qdw + (int64_t)(j + S) * STAGE, QBYTES, &qbw[s]);
                    q_issued = j + S + 1;
                }
            }
            // ---- B^T: contractions in y then x --------------------------------
    #pragma unroll
            for (int c = 0; c < D; ++c) {
                T F0[D][Q], F1[D][Q];
    #pragma unroll
                for (int b = 0; b < D; ++b)
    #pragma unroll
                    for (int qx = 0; qx < Q; ++qx) {
                        T s0 = 0, s1 = 0;
    #pragma unroll
                        for (int qy = 0; qy < Q; ++qy) {
                            if (HK) {
                                s0 += TB::G(P, qy, b) * C1[c][qy][qx];
                                s1 += TB::B(P, qy, b) * C2[c][qy][qx];
                            }
                            s0 += TB::B(P, qy, b) * C0[c][qy][qx];
                        }
                        F0[b][qx] = s0;
                        F1[b][qx] = s1;
                    }
    #pragma unroll
                for (int b = 0; b < D; ++b)
    #pragma unroll
                    for (int a = 0; a < D; ++a) {
                        T s = 0;
    #pragma unroll
                        for (int qx = 0; qx < Q; ++qx) {
                            s += TB::B(P, qx, a) * F0[b][qx];
                            if (HK) s += TB::G(P, qx, a) * F1[b][qx];
                        }
                        out[c][b][a] = s;
                    }
            }
        } else {
            // Q3 (FP32 full format, FP64 both formats): slab sum factorisation.
            // The element's 64 values and its 3 x 64 gradient intermediates do
            // not fit the register file together in FP64, so the quadrature
            // points are taken one qy slab (QH of its Q columns) at a time: the y
            // contraction of the element values (read from the shared-memory x
            // tile) for this qy, then x, then per column z, D and z^T, then the
            // transposed x and y of the slab into the element result.  With
            // QH = Q every contraction is done once (the flop count of the full
            // sum factorisation, slab state 3 x Q x Q values); QH = Q/2 repeats
            // the y contractions once per half slab for a smaller state.  The
            // column order and the data read per column are those of the stream.
#pragma unroll
            for (int c = 0; c < D; ++c)
#pragma unroll
                for (int b = 0; b < D; ++b)
#pragma unroll
                    for (int a = 0; a < D; ++a) out[c][b][a] = T(0);
            // (a per-element branch around the mask measured slower than the
            // predicated form: it splits the unrolled code in two)
            const T *xe = xt + (warp * P) * XW + lane * P;
            auto uval = [&](int c, int b, int a) -> T {
                const T v = xe[(c * RY + b) * XW + a];
                const bool e = (a == 0 && fx0) || (a == P && fx1) || (b == 0 && fy0) || (b == P && fy1) ||
                               (c == 0 && fz0) || (c == P && fz1);
                return e ? T(0) : v;
            };
            constexpr int QH = (sizeof(T) == 8 && FMT == 0) ? FG_Q3_QH : Q;
            static_assert(Q % QH == 0, "slab width must divide Q");
            T Ge[6] = {0, 0, 0, 0, 0, 0};
            const T *ql = nullptr;
            if (FMT == 1) {
                const int j = lz, s = j % S;
                wait_stage(&qbw[s], (j / S) & 1, A.err, wlim, ok, q_waited, j + 1);
                ql = qsw + s * STAGE;
#pragma unroll
                for (int k = 0; k < NCE; ++k) Ge[k] = ql[k * 32 + lane];
            }
#pragma unroll 1
            for (int qy = 0; qy < Q; ++qy) {
                T by[D], gyb[D];
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    by[k] = TB::B(P, qy, k);
                    gyb[k] = TB::G(P, qy, k);
                }
#pragma unroll
                for (int h0 = 0; h0 < Q; h0 += QH) {
                    // forward: y (this qy) then x, per z layer c -> slab [c][qx - h0]
                    T C0[D][QH], C1[D][QH], C2[D][QH];
#pragma unroll
                    for (int c = 0; c < D; ++c) {
                        T R[D], Rg[D];
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            T s0 = 0, s1 = 0;
#pragma unroll
                            for (int b = 0; b < D; ++b) {
                                const T u = uval(c, b, a);
                                s0 += by[b] * u;
                                if (HK) s1 += gyb[b] * u;
                            }
                            R[a] = s0;
                            Rg[a] = s1;
                        }
#pragma unroll
                        for (int k = 0; k < QH; ++k) {
                            const int qx = h0 + k;
                            T t0 = 0, t1 = 0, t2 = 0;
#pragma unroll
                            for (int a = 0; a < D; ++a) {
                                t0 += TB::B(P, qx, a) * R[a];
                                if (HK) {
                                    t1 += TB::B(P, qx, a) * Rg[a];
                                    t2 += TB::G(P, qx, a) * R[a];
                                }
                            }
                            C0[c][k] = t0;
                            C1[c][k] = t1;
                            C2[c][k] = t2;
                        }
                    }
                    // per column of the slab: z, D, z^T (in place)
#pragma unroll
                    for (int k = 0; k < QH; ++k) {
                        const int qx = h0 + k;
                        const int col = qy * Q + qx;
                        const int j = lz * COLS + col;
                        const int s = j % S;
                        if (FMT == 0) {
                            wait_stage(&qbw[s], (j / S) & 1, A.err, wlim, ok, q_waited, j + 1);
                        }
                        const T *qc = FMT == 0 ? qsw + s * STAGE : ql;
                        T vx[Q], vy[Q], vz[Q], vu[Q];
#pragma unroll
                        for (int qz = 0; qz < Q; ++qz) {
                            T gx = 0, gy = 0, gz = 0, ui = 0;
#pragma unroll
                            for (int c = 0; c < D; ++c) {
                                if (HK) {
                                    gx += TB::B(P, qz, c) * C2[c][k];
                                    gy += TB::B(P, qz, c) * C1[c][k];
                                    gz += TB::G(P, qz, c) * C0[c][k];
                                }
                                if (HM) ui += TB::B(P, qz, c) * C0[c][k];
                            }
                            vx[qz] = vy[qz] = vz[qz] = vu[qz] = T(0);
                            if (FMT == 0) {
                                const T *qq = qc + qz * (NC * 32) + lane;
                                if (HK) {
                                    const T d0 = qq[0], d1 = qq[32], d2 = qq[64], d3 = qq[96], d4 = qq[128], d5 = qq[160];
                                    vx[qz] = d0 * gx + d1 * gy + d2 * gz;
                                    vy[qz] = d1 * gx + d3 * gy + d4 * gz;
                                    vz[qz] = d2 * gx + d4 * gy + d5 * gz;
                                }
                                if (HM) vu[qz] = qq[(HK ? 6 : 0) * 32] * ui;
                            } else {
                                const T *qq = qc + (NCE + (col * Q + qz) * NCQ) * 32 + lane;
                                if (HK) {
                                    const T sk = qq[0];
                                    const T hx = sk * gx, hy = sk * gy, hz = sk * gz;
                                    vx[qz] = Ge[0] * hx + Ge[1] * hy + Ge[2] * hz;
                                    vy[qz] = Ge[1] * hx + Ge[3] * hy + Ge[4] * hz;
                                    vz[qz] = Ge[2] * hx + Ge[4] * hy + Ge[5] * hz;
                                }
                                if (HM) vu[qz] = qq[(HK ? 1 : 0) * 32] * ui;
                            }
                        }
#pragma unroll
                        for (int c = 0; c < D; ++c) {
                            T e0 = 0, e1 = 0, e2 = 0;
#pragma unroll
                            for (int qz = 0; qz < Q; ++qz) {
                                if (HK) {
                                    e2 += TB::B(P, qz, c) * vx[qz];
                                    e1 += TB::B(P, qz, c) * vy[qz];
                                    e0 += TB::G(P, qz, c) * vz[qz];
                                }
                                if (HM) e0 += TB::B(P, qz, c) * vu[qz];
                            }
                            C0[c][k] = e0;
                            C1[c][k] = e1;
                            C2[c][k] = e2;
                        }
                        if (FMT == 0) {
                            __syncwarp();
                            if (lane == 0 && ok && j + S < total_cols) {
                                fence_proxy_async();
                                mbar_arrive_expect_tx(&qbw[s], QBYTES);
                                bulk_g2s(qsw + s * STAGE, qdw + (int64_t)(j + S) * STAGE, QBYTES, &qbw[s]);
                                q_issued = j + S + 1;
                            }
                        }
                    }
                    // transposed x then y of the slab into the element result
#pragma unroll
                    for (int c = 0; c < D; ++c) {
                        T H0[D], H1[D];
#pragma unroll
                        for (int a = 0; a < D; ++a) {
                            T s0 = 0, s1 = 0;
#pragma unroll
                            for (int k = 0; k < QH; ++k) {
                                const int qx = h0 + k;
                                s0 += TB::B(P, qx, a) * C0[c][k];
                                if (HK) {
                                    s0 += TB::G(P, qx, a) * C2[c][k];
                                    s1 += TB::B(P, qx, a) * C1[c][k];
                                }
                            }
                            H0[a] = s0;
                            H1[a] = s1;
                        }
#pragma unroll
                        for (int b = 0; b < D; ++b)
#pragma unroll
                            for (int a = 0; a < D; ++a) {
                                T v = out[c][b][a] + by[b] * H0[a];
                                if (HK) v += gyb[b] * H1[a];
                                out[c][b][a] = v;
                            }
                    }
                }
            }
            if (FMT == 1) {
                const int j = lz, s = j % S;
                __syncwarp();
                if (lane == 0 && ok && j + S < total_cols) {
                    fence_proxy_async();
                    mbar_arrive_expect_tx(&qbw[s], QBYTES);
                    bulk_g2s(qsw + s * STAGE, qdw + (int64_t)(j + S) * STAGE, QBYTES, &qbw[s]);
                    q_issued = j + S + 1;
                }
            }
        }
        // ---- E^T: merge + store --------------------------------------------
        merge_and_store<P, T, WY>(
            out, g, ybuf, carry, lz, nl, tz, warp, lane, item, valid, lane_last, w_last, fx0, fx1,
            fy0, fy1, fz0, fz1, A.y, A.face, A.accumulate,
            [&](int c, int b, int a) { return xt[(c * RY + warp * P + b) * XW + lane * P + a]; });
        __syncthreads();
    }
    // After a timeout, drain the copies this thread issued and has not seen
    // arrive (the one whose wait ran out included), with bounded waits.
    if (!ok) {
        if (lane == 0) drain_stages(qbw, S, q_waited, q_issued);
        if (threadIdx.x == 0) drain_stages(xbar, SM::NXB, x_waited, x_issued);
    }
    if (A.fixcnt)  // the y staging area is free after the last layer's barrier
        fused_fixup<T, P>(g, A.y, A.face, A.fixcnt, item, reinterpret_cast<int *>(ybuf));
}

// Single operator: one CTA per item; the x tile map is a kernel parameter.
template <int P, int OPK, typename T, int WY, int S, int MINB, int FMT = 0>
__global__ void __launch_bounds__(WY * 32, MINB)
    pa_apply_kernel(const __grid_constant__ CUtensorMap xmap, const ApplyArgs<T> A) {
    pa_apply_body<P, OPK, T, WY, S, FMT>(&xmap, A, A.item0 + blockIdx.x);
}

// Batched operators (many independent instances of the same order, kind and
// format in one launch): block b works on item bmap[b].y of instance
// bmap[b].x; each instance's arguments and x tile maps (one per input slot,
// encoded once per batch, 64-byte aligned in global memory) come from tables.
template <typename T> struct BatchApply {
    const ApplyArgs<T> *args;    // [instance][slot]
    const CUtensorMap *tmaps;    // [instance][slot]
    const int2 *bmap;            // [block] -> (instance, item)
    int nslots, slot;
};
template <int P, int OPK, typename T, int WY, int S, int MINB, int FMT = 0>
__global__ void __launch_bounds__(WY * 32, MINB) pa_apply_batched_kernel(const BatchApply<T> B) {
    const int2 m = B.bmap[blockIdx.x];
    const int k = m.x * B.nslots + B.slot;
    pa_apply_body<P, OPK, T, WY, S, FMT>(&B.tmaps[k], B.args[k], m.y);
}

// ---------------------------------------------------------------------------
// Diagonal of the operator (Jacobi).  Same item decomposition and scatter; the
// element diagonal sum_q g_i^T D_q g_i (+ m_q phi_i^2) is formed directly from
// the quadrature data in global memory (a setup-time kernel).
// ---------------------------------------------------------------------------
template <int P, int OPK, typename T, int WY>
__global__ void __launch_bounds__(WY * 32) pa_diag_kernel(const ApplyArgs<T> A) {
    constexpr int D = P + 1, Q = P + 1, NC = NComp<OPK>::v;
    constexpr bool HM = (OPK & 1) != 0, HK = (OPK & 2) != 0;
    using TB = Tab<T>;
    const Grid g = A.g;
    __shared__ T ybuf[WY * D * D * 32];
    __shared__ T carry[D * D * WY * 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int item = blockIdx.x;
    const int tx = item % g.ntx, ty = (item / g.ntx) % g.nty, tz = item / (g.ntx * g.nty);
    const int nl = min(g.TZ, g.nz - tz * g.TZ);
    const int ex = tx * 32 + lane, ey = ty * WY + warp;
    const bool valid = ex < g.nx && ey < g.ny;
    const int lane_last = min(31, g.nx - 1 - tx * 32);
    const int w_last = min(WY - 1, g.ny - 1 - ty * WY);
    const int ess = g.ess;
    const bool fx0 = (ess & 16) && ex == 0, fx1 = (ess & 32) && ex == g.nx - 1;
    const bool fy0 = (ess & 4) && ey == 0, fy1 = (ess & 8) && ey == g.ny - 1;
    for (int lz = 0; lz < nl; ++lz) {
        const int ez = tz * g.TZ + lz;
        const bool fz0 = (ess & 1) && ez == 0, fz1 = (ess & 2) && ez == g.nz - 1;
        T out[D][D][D];
#pragma unroll
        for (int c = 0; c < D; ++c)
#pragma unroll
            for (int b = 0; b < D; ++b)
#pragma unroll
                for (int a = 0; a < D; ++a) out[c][b][a] = 0;
        for (int qz = 0; qz < Q; ++qz)
            for (int qy = 0; qy < Q; ++qy)
#pragma unroll
                for (int qx = 0; qx < Q; ++qx) {
                    const T *qq = A.qd + qd_index<P, OPK>(g, item, warp, lz, qy * Q + qx, qz, 0, lane);
                    T d[7];
#pragma unroll
                    for (int k = 0; k < NC; ++k) d[k] = qq[k * 32];
#pragma unroll
                    for (int c = 0; c < D; ++c)
#pragma unroll
                        for (int b = 0; b < D; ++b)
#pragma unroll
                            for (int a = 0; a < D; ++a) {
                                const T Bx = TB::B(P, qx, a), By = TB::B(P, qy, b), Bz = TB::B(P, qz, c);
                                T s = 0;
                                if (HK) {
                                    const T gx = TB::G(P, qx, a) * By * Bz;
                                    const T gy = Bx * TB::G(P, qy, b) * Bz;
                                    const T gz = Bx * By * TB::G(P, qz, c);
                                    s = d[0] * gx * gx + d[3] * gy * gy + d[5] * gz * gz +
                                        T(2) * (d[1] * gx * gy + d[2] * gx * gz + d[4] * gy * gz);
                                }
                                if (HM) {
                                    const T ph = Bx * By * Bz;
                                    s += d[HK ? 6 : 0] * ph * ph;
                                }
                                out[c][b][a] += s;
                            }
                }
        merge_and_store<P, T, WY>(out, g, ybuf, carry, lz, nl, tz, warp, lane, item, valid,
                                  lane_last, w_last, fx0, fx1, fy0, fy1, fz0, fz1, A.y, A.face, 0,
                                  [](int, int, int) { return T(1); });
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Fix-up: for every DOF on an item's lower face that a neighbour item also
// touches, add the neighbours' face-slot partials to the owner's value, in a
// fixed (dz, dy, dx) order.  The work is split into rows of DOFs on the shared
// planes (fixup_rows).  x planes own all their DOFs, y planes skip DOFs on x
// planes, z planes skip DOFs on x or y planes.  32-bit index arithmetic except
// the DOF offset.
// ---------------------------------------------------------------------------
template <bool CG, typename T> __device__ __forceinline__ T ld_face(const T *p) {
    if constexpr (CG) return __ldcg(p);  // written by other CTAs of the same launch: read at L2
    else return *p;
}

// The neighbours' face-slot partials of one shared DOF added to `own` in
// (dz, dy, dx) order.  (tx, ty, tz): the owner item; (sx, sy, sz): whether the
// DOF lies on an x / y / z plane between items.  CG: loads at L2 (the fused
// fix-up reads slots other CTAs of the same launch wrote).
template <typename T, bool CG = false>
__device__ __forceinline__ T fixup_acc(const Grid &g, int I, int J, int K, int tx, int ty, int tz,
                                       int sx, int sy, int sz, T own, const T *__restrict__ face) {
    const int SXe = 32 * g.p, SYe = g.WY * g.p, SZe = g.TZ * g.p;
    const int fs = g.face_stride(), fxs = g.fx(), fys = g.fy();
    T sum = own;
    for (int dz = 0; dz <= sz; ++dz)
        for (int dy = 0; dy <= sy; ++dy)
            for (int dx = 0; dx <= sx; ++dx) {
                if (!(dx | dy | dz)) continue;
                const int nx_ = tx - dx, ny_ = ty - dy, nz_ = tz - dz;
                const int nb = (nz_ * g.nty + ny_) * g.ntx + nx_;
                const int I0 = nx_ * SXe, J0 = ny_ * SYe, K0 = nz_ * SZe;
                const T *fb = face + (int64_t)nb * fs;
                if (dx)
                    sum += ld_face<CG>(fb + (K - K0) * (SYe + 1) + (J - J0));
                else if (dy)
                    sum += ld_face<CG>(fb + fxs + (K - K0) * (SXe + 1) + (I - I0));
                else
                    sum += ld_face<CG>(fb + fxs + fys + (J - J0) * (SXe + 1) + (I - I0));
            }
    return sum;
}

// Rows of shared-face DOFs: the x planes as NK rows of NJ DOFs (u -> J), the
// y planes as NK rows of NI DOFs (u -> I), the z planes as NJ rows of NI DOFs
// (u -> I); x planes first, then y, then z.
__host__ __device__ inline int fixup_rows(const Grid &g) {
    return (g.ntx - 1) * g.NK + (g.nty - 1) * g.NK + (g.ntz - 1) * g.NJ;
}

// One row of the fix-up, by the whole block.  Everything fixed along the row
// (its plane, the owner item across the plane, the essential faces it lies on)
// is worked out once; per DOF only the position along the row is classified,
// by a division by the compile-time 32 P.  A DOF (I, J, K) with sx = (0 < I < NI-1
// and I % 32P == 0), sy, sz alike, owned by item (min(I / 32P, ntx-1), ...), gets
// the sum of fixup_acc.  y planes skip DOFs on x planes, z planes skip DOFs on x or
// y planes; essential DOFs keep the owner's value.
template <typename T, int P>
__device__ __forceinline__ void fixup_row_t(const Grid &g, int r, T *__restrict__ y,
                                            const T *__restrict__ face) {
    constexpr int SXe = 32 * P;
    const int SYe = g.WY * P, SZe = g.TZ * P;
    const int rx = (g.ntx - 1) * g.NK, ry = (g.nty - 1) * g.NK;
    const int ess = g.ess;
    if (r < rx) {  // x plane I = (pl + 1) SXe; u -> J, row -> K
        const int pl = r / g.NK, K = r - pl * g.NK, I = (pl + 1) * SXe, tx = pl + 1;
        if (((ess & 1) && K == 0) || ((ess & 2) && K == g.NK - 1)) return;
        const int sz = (K > 0 && K < g.NK - 1 && K % SZe == 0), tz = min(K / SZe, g.ntz - 1);
        T *yr = y + (int64_t)K * g.NJ * g.NIp + I;
        for (int J = threadIdx.x; J < g.NJ; J += blockDim.x) {
            if (((ess & 4) && J == 0) || ((ess & 8) && J == g.NJ - 1)) continue;
            const int sy = (J > 0 && J < g.NJ - 1 && J % SYe == 0), ty = min(J / SYe, g.nty - 1);
            T *yp = yr + (int64_t)J * g.NIp;
            *yp = fixup_acc<T>(g, I, J, K, tx, ty, tz, 1, sy, sz, *yp, face);
        }
    } else if (r < rx + ry) {  // y plane J = (pl + 1) SYe; u -> I, row -> K
        r -= rx;
        const int pl = r / g.NK, K = r - pl * g.NK, J = (pl + 1) * SYe, ty = pl + 1;
        if (((ess & 1) && K == 0) || ((ess & 2) && K == g.NK - 1)) return;
        const int sz = (K > 0 && K < g.NK - 1 && K % SZe == 0), tz = min(K / SZe, g.ntz - 1);
        T *yr = y + ((int64_t)K * g.NJ + J) * g.NIp;
        for (int I = threadIdx.x; I < g.NI; I += blockDim.x) {
            const int q = I / SXe;
            if (I > 0 && I < g.NI - 1 && I == q * SXe) continue;  // on an x plane
            if (((ess & 16) && I == 0) || ((ess & 32) && I == g.NI - 1)) continue;
            yr[I] = fixup_acc<T>(g, I, J, K, min(q, g.ntx - 1), ty, tz, 0, 1, sz, yr[I], face);
        }
    } else {  // z plane K = (pl + 1) SZe; u -> I, row -> J
        r -= rx + ry;
        const int pl = r / g.NJ, J = r - pl * g.NJ, K = (pl + 1) * SZe, tz = pl + 1;
        if (J > 0 && J < g.NJ - 1 && J % SYe == 0) return;  // on a y plane
        if (((ess & 4) && J == 0) || ((ess & 8) && J == g.NJ - 1)) return;
        const int ty = min(J / SYe, g.nty - 1);
        T *yr = y + ((int64_t)K * g.NJ + J) * g.NIp;
        for (int I = threadIdx.x; I < g.NI; I += blockDim.x) {
            const int q = I / SXe;
            if (I > 0 && I < g.NI - 1 && I == q * SXe) continue;  // on an x plane
            if (((ess & 16) && I == 0) || ((ess & 32) && I == g.NI - 1)) continue;
            yr[I] = fixup_acc<T>(g, I, J, K, min(q, g.ntx - 1), ty, tz, 0, 0, 1, yr[I], face);
        }
    }
}

template <typename T>
__device__ __forceinline__ void fixup_row(const Grid &g, int r, T *__restrict__ y,
                                          const T *__restrict__ face) {
    switch (g.p) {
    case 1: fixup_row_t<T, 1>(g, r, y, face); break;
    case 2: fixup_row_t<T, 2>(g, r, y, face); break;
    default: fixup_row_t<T, 3>(g, r, y, face); break;
    }
}

// The shared DOFs owned by item (ox, oy, oz): those on its lower x, y and z
// faces that a lower neighbour item also touches (the same DOFs, owner and
// plane flags as the rows of fixup_row_t), fixed up by the whole block.
template <typename T, int P>
__device__ __forceinline__ void fixup_owner(const Grid &g, T *y, const T *face, int ox, int oy,
                                            int oz) {
    constexpr int SXe = 32 * P;
    const int SYe = g.WY * P, SZe = g.TZ * P;
    const int I0 = ox * SXe, J0 = oy * SYe, K0 = oz * SZe;
    const int I1 = ox == g.ntx - 1 ? g.NI - 1 : I0 + SXe - 1;
    const int J1 = oy == g.nty - 1 ? g.NJ - 1 : J0 + SYe - 1;
    const int K1 = oz == g.ntz - 1 ? g.NK - 1 : K0 + SZe - 1;
    const int ia = I0 + (ox > 0), ja = J0 + (oy > 0);  // first I / J off the owner's x / y plane
    const int nI = I1 - ia + 1, nJ = J1 - J0 + 1, nJy = J1 - ja + 1, nK = K1 - K0 + 1;
    const int cx = ox > 0 ? nJ * nK : 0;   // x face (J, K)
    const int cy = oy > 0 ? nI * nK : 0;   // y face (I, K), off the x plane
    const int cz = oz > 0 ? nI * nJy : 0;  // z face (I, J), off the x and y planes
    for (int t = threadIdx.x; t < cx + cy + cz; t += blockDim.x) {
        int I, J, K, sx, sy, sz;
        if (t < cx) {
            const int k = t / nJ;
            J = J0 + (t - k * nJ); K = K0 + k; I = I0;
            sx = 1; sy = (J == J0 && oy > 0); sz = (K == K0 && oz > 0);
        } else if (t < cx + cy) {
            const int u = t - cx, k = u / nI;
            I = ia + (u - k * nI); K = K0 + k; J = J0;
            sx = 0; sy = 1; sz = (K == K0 && oz > 0);
        } else {
            const int u = t - cx - cy, j = u / nI;
            I = ia + (u - j * nI); J = ja + j; K = K0;
            sx = 0; sy = 0; sz = 1;
        }
        if (g.is_ess(I, J, K)) continue;
        T *yp = y + g.dof(I, J, K);
        *yp = fixup_acc<T, true>(g, I, J, K, ox, oy, oz, sx, sy, sz, __ldcg(yp), face);
    }
}

// Fix-up fused into the apply (a run-time option, off by default: measured
// slower than fixup_kernel, 0.657 against 0.503 ms for the 128^3 Q2 FP64
// apply, because the last arriver's owner fix-up is a serial tail of
// L2-latency-bound loads on an SM slot that would otherwise stream qdata).
// Once an item has stored its values and face slots it arrives at the counter
// of every item whose lower faces it touches (itself and its upper neighbours
// in x, y and z).  The last of an owner's contributors to arrive (an arrival
// count, not a wait: no CTA waits on another) resets the owner's counter for
// the next launch and adds the face partials into the owner's lower-face DOFs:
// the sums of fixup_acc in the same order, so the result is bit-identical to
// fixup_kernel's.  `flag` is one int of shared memory that is free at this
// point.
template <typename T, int P>
__device__ __forceinline__ void fused_fixup(const Grid &g, T *y, const T *face, unsigned *cnt,
                                            int item, int *flag) {
    const int tx = item % g.ntx, ty = (item / g.ntx) % g.nty, tz = item / (g.ntx * g.nty);
    __threadfence();  // this thread's y and face-slot stores, before the arrival below
    __syncthreads();
    for (int o = 0; o < 8; ++o) {
        const int ox = tx + (o & 1), oy = ty + ((o >> 1) & 1), oz = tz + (o >> 2);
        if (ox >= g.ntx || oy >= g.nty || oz >= g.ntz) continue;
        const unsigned need = (1u + (ox > 0)) * (1u + (oy > 0)) * (1u + (oz > 0));
        if (need == 1u) continue;  // no lower neighbour: nothing shared below
        const int owner = (oz * g.nty + oy) * g.ntx + ox;
        if (threadIdx.x == 0) {
            const unsigned prev = atomicAdd(&cnt[owner], 1u);
            const int last = prev == need - 1u;
            if (last) {
                atomicExch(&cnt[owner], 0u);
                __threadfence();  // the contributors' stores, before this block reads them
            }
            *flag = last;
        }
        __syncthreads();
        const int last = *flag;
        __syncthreads();
        if (last) fixup_owner<T, P>(g, y, face, ox, oy, oz);
    }
}

// One block per row of shared-face DOFs (grid = fixup_rows(g)).
template <typename T>
__global__ void __launch_bounds__(128) fixup_kernel(const Grid g, T *__restrict__ y,
                                                    const T *__restrict__ face, const int *skip) {
    if (skip && *skip) return;
    fixup_row<T>(g, blockIdx.x, y, face);
}

// Fix-up of the shared DOFs owned by the DOF planes [Ka, Kb): the x- and
// y-plane rows of those planes and the z-plane rows of the item-layer
// boundaries pl0 .. pl0 + npl - 1 inside the range, in fixup_row's numbering
// (used when an apply is run one range of item layers at a time).
template <typename T>
__global__ void __launch_bounds__(128) fixup_range_kernel(const Grid g, T *__restrict__ y,
                                                          const T *__restrict__ face, int Ka, int Kb, int pl0) {
    const int nk = Kb - Ka;
    const int rx = (g.ntx - 1) * nk, ry = (g.nty - 1) * nk;
    int b = blockIdx.x, r;
    if (b < rx) {
        r = (b / nk) * g.NK + Ka + b % nk;
    } else if (b < rx + ry) {
        b -= rx;
        r = (g.ntx - 1) * g.NK + (b / nk) * g.NK + Ka + b % nk;
    } else {
        b -= rx + ry;
        r = (g.ntx - 1) * g.NK + (g.nty - 1) * g.NK + (pl0 + b / g.NJ) * g.NJ + b % g.NJ;
    }
    fixup_row<T>(g, r, y, face);
}

// Batched fix-up: blockIdx.y = instance; blocks stride over the instance's
// rows of shared-face DOFs.
template <typename T> struct FixArgs {
    Grid g;
    T *y;
    const T *face;
    const int *skip;
};
template <typename T>
__global__ void __launch_bounds__(128) fixup_batched_kernel(const FixArgs<T> *args, int nslots,
                                                            int slot) {
    const FixArgs<T> &A = args[blockIdx.y * nslots + slot];
    if (A.skip && *A.skip) return;
    const int rows = fixup_rows(A.g);
    for (int r = blockIdx.x; r < rows; r += gridDim.x) fixup_row<T>(A.g, r, A.y, A.face);
}

// ---------------------------------------------------------------------------
// Quadrature-data setup: one thread per (element, quadrature point).
// Trilinear geometry from the 8 element vertices (HexQ1 node order of
// crates/element/src/lagrange/hex.rs:27-36), J_id = sum_k x_k[i] dphi_k/dxi_d
// (assembler.rs:96-123), D = w |detJ| kappa c_k J^-1 J^-T, m = w |detJ| rho c_m.
// ---------------------------------------------------------------------------
struct SetupArgs {
    Grid g;
    const double *vcoord;   // (nx+1)(ny+1)(nz+1)*3 or null (uniform unit cube)
    const double *kappa_q;  // [E][qz][qy][qx] or null
    const double *rho_q;
    double kappa_c, rho_c, c_m, c_k;
    double gx[4], gw[4];    // Gauss rule for Q = p+1 points
    int *err;
};

// Re-layout of full-format quadrature data for another z extent of the items
// (TZ): the data of element e, point (col, qz), component c moves from its
// place under grid go to its place under grid gn (same mesh, same WY).  One
// thread per (element, point); pads of the new layout stay as initialised.
template <int P, int OPK>
__global__ void qdata_relayout_kernel(const Grid go, const Grid gn, const double *__restrict__ src,
                                      double *__restrict__ dst) {
    constexpr int Q = P + 1, NC = NComp<OPK>::v;
    const int64_t total = (int64_t)go.nx * go.ny * go.nz * Q * Q * Q;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int cq = (int)(t % (Q * Q * Q));
        const int64_t e = t / (Q * Q * Q);
        const int col = cq / Q, qz = cq % Q;
        const int ex = (int)(e % go.nx), ey = (int)((e / go.nx) % go.ny), ez = (int)(e / ((int64_t)go.nx * go.ny));
        const int tx = ex / 32, lane = ex % 32, ty = ey / go.WY, wy = ey % go.WY;
        const int io = ((ez / go.TZ) * go.nty + ty) * go.ntx + tx, lo = ez % go.TZ;
        const int in = ((ez / gn.TZ) * gn.nty + ty) * gn.ntx + tx, ln = ez % gn.TZ;
        const double *s = src + qd_index<P, OPK>(go, io, wy, lo, col, qz, 0, lane);
        double *d = dst + qd_index<P, OPK>(gn, in, wy, ln, col, qz, 0, lane);
#pragma unroll
        for (int c = 0; c < NC; ++c) d[c * 32] = s[c * 32];
    }
}

// Affine-compressed quadrature data (FMT 1) derived from the full FP64 data:
// on an element with constant J every D_q is w_q kappa_q times the same
// symmetric matrix |detJ| J^-1 J^-T, so G_e = D_{q0} and s_q = tr(D_q)/tr(D_{q0})
// reproduce D_q = s_q G_e.  Each thread (element, quadrature point) checks
// that identity to 1e-10 relative and raises FG_DERR_BOUNDS otherwise (the
// mesh is not affine: the format is refused).  The mass scalar is copied.
template <int P, int OPK, typename T>
__global__ void qdata_compress_kernel(const Grid g, const double *__restrict__ qfull,
                                      T *__restrict__ qaff, int *err) {
    constexpr int Q = P + 1, NC = NComp<OPK>::v;
    constexpr bool HM = (OPK & 1) != 0, HK = (OPK & 2) != 0;
    constexpr int NCE = AffineComp<OPK>::NCE, NCQ = AffineComp<OPK>::NCQ;
    constexpr int STG = stage_elems<P, OPK, 1>();
    const int64_t E = (int64_t)g.nx * g.ny * g.nz;
    const int64_t total = E * Q * Q * Q;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int q = (int)(t % (Q * Q * Q));
        const int64_t e = t / (Q * Q * Q);
        const int qx = q % Q, qy = (q / Q) % Q, qz = q / (Q * Q);
        const int ex = (int)(e % g.nx), ey = (int)((e / g.nx) % g.ny), ez = (int)(e / ((int64_t)g.nx * g.ny));
        const int tx = ex / 32, lane = ex % 32, ty = ey / g.WY, wy = ey % g.WY, tz = ez / g.TZ,
                  lz = ez % g.TZ;
        const int item = (tz * g.nty + ty) * g.ntx + tx;
        const int col = qy * Q + qx;
        const double *src = qfull + qd_index<P, OPK>(g, item, wy, lz, col, qz, 0, lane);
        const double *src0 = qfull + qd_index<P, OPK>(g, item, wy, lz, 0, 0, 0, lane);
        T *base = qaff + ((((int64_t)item * g.WY + wy) * g.TZ + lz) * STG) + lane;
        T *qq = base + (NCE + (col * Q + qz) * NCQ) * 32;
        if (HK) {
            const double tr = src[0] + src[96] + src[160];
            const double tr0 = src0[0] + src0[96] + src0[160];
            const double sq = tr0 != 0.0 ? tr / tr0 : 0.0;
            double nrm = 0.0, dif = 0.0;
            for (int k = 0; k < 6; ++k) {
                nrm = fmax(nrm, fabs(src[k * 32]));
                dif = fmax(dif, fabs(src[k * 32] - sq * src0[k * 32]));
            }
            if (dif > 1e-10 * nrm && err) atomicOr(err, FG_DERR_BOUNDS);
            qq[0] = (T)sq;
            if (q == 0)
                for (int k = 0; k < 6; ++k) base[k * 32] = (T)src0[k * 32];
        }
        if (HM) qq[(HK ? 1 : 0) * 32] = (T)src[(HK ? 6 : 0) * 32];
        (void)NC;
    }
}

// Quadrature data of one point from the element's 8 vertices xv (HexQ1 node
// order of crates/element/src/lagrange/hex.rs:27-36) at the reference point xi
// with weight w: J_id = sum_k x_k[i] dphi_k/dxi_d (assembler.rs:96-123),
// D = w |detJ| kappa c_k J^-1 J^-T (6 symmetric components xx xy xz yy yz zz),
// m = w |detJ| rho c_m.  Returns false when det J = 0.
__device__ __forceinline__ bool hex_point_qdata(const double (&xv)[8][3], const double (&xi)[3], double w,
                                                double kap, double c_k, double rho, double c_m, double (&D)[6],
                                                double &m) {
    const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                           {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int k = 0; k < 8; ++k) {
        const double sx = off[k][0] ? 1.0 : -1.0, sy = off[k][1] ? 1.0 : -1.0, sz = off[k][2] ? 1.0 : -1.0;
        const double fx = 1.0 + sx * xi[0], fy = 1.0 + sy * xi[1], fz = 1.0 + sz * xi[2];
        const double gr[3] = {0.125 * sx * fy * fz, 0.125 * sy * fx * fz, 0.125 * sz * fx * fy};
        for (int i = 0; i < 3; ++i)
            for (int d = 0; d < 3; ++d) J[i][d] += xv[k][i] * gr[d];
    }
    const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                       J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                       J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    const double wd = w * fabs(det);
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
    const double s = wd * kap * c_k;
    const int mi[6] = {0, 0, 0, 1, 1, 2}, ni[6] = {0, 1, 2, 1, 2, 2};
    for (int k = 0; k < 6; ++k) {
        const int a = mi[k], b = ni[k];
        D[k] = s * (inv[a][0] * inv[b][0] + inv[a][1] * inv[b][1] + inv[a][2] * inv[b][2]);
    }
    m = wd * rho * c_m;
    return fabs(det) > 0.0;
}

template <int P, int OPK, typename T>
__global__ void qdata_setup_kernel(const SetupArgs S, T *__restrict__ qd) {
    constexpr int Q = P + 1, NC = NComp<OPK>::v;
    constexpr bool HM = (OPK & 1) != 0, HK = (OPK & 2) != 0;
    const Grid &g = S.g;
    const int64_t E = (int64_t)g.nx * g.ny * g.nz;
    const int64_t total = E * Q * Q * Q;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int q = (int)(t % (Q * Q * Q));
        const int64_t e = t / (Q * Q * Q);
        const int qx = q % Q, qy = (q / Q) % Q, qz = q / (Q * Q);
        const int ex = (int)(e % g.nx), ey = (int)((e / g.nx) % g.ny), ez = (int)(e / ((int64_t)g.nx * g.ny));
        const double xi[3] = {S.gx[qx], S.gx[qy], S.gx[qz]};
        const double w = S.gw[qx] * S.gw[qy] * S.gw[qz];
        const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                               {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
        double xv[8][3];
        for (int k = 0; k < 8; ++k) {
            const int vi = ex + off[k][0], vj = ey + off[k][1], vk = ez + off[k][2];
            if (S.vcoord) {
                const int64_t id = ((int64_t)vk * (g.ny + 1) + vj) * (g.nx + 1) + vi;
                xv[k][0] = S.vcoord[3 * id];
                xv[k][1] = S.vcoord[3 * id + 1];
                xv[k][2] = S.vcoord[3 * id + 2];
            } else {
                xv[k][0] = (double)vi / g.nx;
                xv[k][1] = (double)vj / g.ny;
                xv[k][2] = (double)vk / g.nz;
            }
        }
        const double kap = S.kappa_q ? S.kappa_q[e * (Q * Q * Q) + q] : S.kappa_c;
        const double rho = S.rho_q ? S.rho_q[e * (Q * Q * Q) + q] : S.rho_c;
        double D[6], m;
        if (!hex_point_qdata(xv, xi, w, kap, S.c_k, rho, S.c_m, D, m) && S.err) atomicOr(S.err, FG_DERR_BOUNDS);
        const int tx = ex / 32, lane = ex % 32, ty = ey / g.WY, wy = ey % g.WY, tz = ez / g.TZ,
                  lz = ez % g.TZ;
        const int item = (tz * g.nty + ty) * g.ntx + tx;
        T *dst = qd + qd_index<P, OPK>(g, item, wy, lz, qy * Q + qx, qz, 0, lane);
        if (HK)
            for (int k = 0; k < 6; ++k) dst[k * 32] = (T)D[k];
        if (HM) dst[(HK ? 6 : 0) * 32] = (T)m;
        (void)NC;
    }
}

}  // namespace fg
