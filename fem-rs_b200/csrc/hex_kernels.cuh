// hex_kernels.cuh -- partial-assembly mass / diffusion operator on an
// unstructured Hex8 mesh of order P (Q = P+1 Gauss points per direction): the
// element loop of crates/assembly/src/partial.rs:85-130, 154-208 with the
// Hex8 geometry of crates/assembly/src/assembler.rs:96-143, for any element
// connectivity and any DOF numbering (a DofManager's element maps).
//
// Data layout.  Elements are put in a Morton order of their centroids and cut
// into chunks of CE = WARPS * 32 elements, one CTA each (the last chunk padded
// to whole 32-element warp groups: padding elements have map entries -1 and
// zero quadrature data).
//   dofs [nl][E]         int32 element-to-DOF map, local DOF (c,b,a) at
//                        k = (c*D + b)*D + a (tensor order on the reference cube);
//                        element-major, so a warp reads each entry in one load
//   qd                   quadrature data in each warp's consumption order:
//                        [group][col = qy*Q + qx][qz][comp][lane], comp the 6
//                        symmetric w|detJ| kappa J^-1 J^-T and/or w|detJ| rho.
//                        One column of a 32-element group is a contiguous stage,
//                        streamed into a per-warp ring of shared-memory stages by
//                        1-D bulk copies on mbarriers (bounded waits, drained on
//                        timeout)
//   ess  [N]             essential-DOF mask (constrained applies)
//   emsk [E]             per element, bit k set: local DOF k is essential (the
//                        gather masks with it instead of reading ess per DOF)
//
// Scatter without float atomics and without an element-result array in HBM
// (chunk_plan.h, chunk_scatter.cuh): a CTA puts its element results in shared
// memory and sums each DOF of its chunk's list over the DOF's element slots in
// a fixed order; a DOF owned by the chunk is stored, a DOF shared with other
// chunks gets a partial that chunk_shared_kernel adds in chunk order.  The
// sums are the same from run to run.
//
// Element math: slab sum factorisation (one qy slab of QH quadrature columns
// at a time: y then x contraction of the element values, per column z, D, z^T,
// then the transposed x and y into the element result).  The element values
// are staged in shared memory, one column per thread.
#pragma once
#include "chunk_scatter.cuh"
#include "fg_common.cuh"
#include "pa_kernels.cuh"

namespace fg {

template <typename T> struct HexApply {
    int64_t E, N;          // elements (padded to whole 32-element groups), DOFs
    const int32_t *dofs;   // [nl][E]
    const T *qd;           // per-group streams (layout above)
    const uint8_t *ess;    // [N] or null
    const uint64_t *emsk;  // [E] essential local DOFs (bit k), or null
    const T *x;            // null: diagonal
    T *y;
    int accumulate, constrained;
    const int *skip;       // if non-null and *skip != 0 the kernel returns at once
    int *err;              // device error word
    uint64_t wait_ns;      // limit of each wait for a stage (0: 1 s)
    ChunkLists L;          // chunks of the CTA size
};

// Index of component `comp` of quadrature point (col, qz) of element e.
template <int P, int OPK> __host__ __device__ inline int64_t hex_qd_index(int64_t e, int col, int qz, int comp) {
    constexpr int Q = P + 1, NC = NComp<OPK>::v;
    return (((e >> 5) * (Q * Q) + col) * Q + qz) * (NC * 32) + comp * 32 + (e & 31);
}

// Shared memory (bytes): a region holding first the per-warp quadrature-data
// rings and, after the element phase, the chunk's lists; the element values
// (then results), one column per thread; the ring barriers.
template <int P, int OPK, typename T, int WARPS, int S> struct HexSmem {
    static constexpr int Q = P + 1, NL = (P + 1) * (P + 1) * (P + 1), BS = WARPS * 32;
    static constexpr int STAGE = Q * NComp<OPK>::v * 32;  // elements of one column stage
    static constexpr int RING = WARPS * S * STAGE * (int)sizeof(T);
    static __host__ __device__ int region(int max_nu) {
        const int l = (int)chunk_list_smem(NL, BS, max_nu);
        return round_up(RING > l ? RING : l, 128);
    }
    static __host__ __device__ int off_x(int max_nu) { return region(max_nu); }
    static __host__ __device__ int off_b(int max_nu) { return round_up(off_x(max_nu) + NL * BS * (int)sizeof(T), 8); }
    static __host__ __device__ int bytes(int max_nu) { return off_b(max_nu) + WARPS * S * 8; }
};

template <int P, int OPK, typename T, int WARPS, int S, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) hex_apply_kernel(const HexApply<T> A) {
    constexpr int D = P + 1, Q = P + 1, NL = D * D * D, NC = NComp<OPK>::v, BS = WARPS * 32;
    constexpr bool HM = (OPK & 1) != 0, HK = (OPK & 2) != 0;
    constexpr int QH = (P == 3 && sizeof(T) == 8) ? 2 : Q;  // half slabs bound the Q3 FP64 state
    constexpr int COLS = Q * Q;
    using SM = HexSmem<P, OPK, T, WARPS, S>;
    constexpr int STAGE = SM::STAGE;
    constexpr uint32_t QBYTES = (uint32_t)(STAGE * sizeof(T));
    using TB = Tab<T>;
    extern __shared__ __align__(128) unsigned char hex_smem[];
    if (A.skip && *A.skip) return;
    const int MU = A.L.max_nu;
    T *ring = reinterpret_cast<T *>(hex_smem);
    T *xs = reinterpret_cast<T *>(hex_smem + SM::off_x(MU));
    uint64_t *bars = reinterpret_cast<uint64_t *>(hex_smem + SM::off_b(MU));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
    const int64_t E = A.E;
    const int64_t group = (int64_t)blockIdx.x * WARPS + warp;  // 32-element group of this warp
    const bool wvalid = group * 32 < E;
    const int64_t e = group * 32 + lane;
    const uint64_t wlim = A.wait_ns ? A.wait_ns : 1000000000ull;
    if (threadIdx.x == 0) {
        for (int i = 0; i < WARPS * S; ++i) mbar_init(&bars[i], 1);
        fence_barrier_init();
    }
    __syncthreads();
    T *qsw = ring + warp * S * STAGE;
    uint64_t *qbw = bars + warp * S;
    const T *qdw = A.qd + group * COLS * STAGE;
    int q_issued = 0, q_waited = 0;
    bool ok = true;
    if (wvalid) {
        if (lane == 0) {
            for (int j = 0; j < S && j < COLS; ++j) {
                mbar_arrive_expect_tx(&qbw[j], QBYTES);
                bulk_g2s(qsw + j * STAGE, qdw + (int64_t)j * STAGE, QBYTES, &qbw[j]);
                q_issued = j + 1;
            }
        }
        // gather (E) with the essential columns masked; padding elements hold -1
        const bool evalid = __ldg(A.dofs + e) >= 0;
        const uint64_t m = (A.constrained && A.emsk) ? __ldg(A.emsk + e) : 0ull;
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            T v = T(0);
            if (evalid) {
                const T xv = __ldg(A.x + __ldg(A.dofs + (int64_t)k * E + e));
                v = ((m >> k) & 1ull) ? T(0) : xv;
            }
            xs[k * BS + tid] = v;
        }
        auto uval = [&](int c, int b, int a) -> T { return xs[((c * D + b) * D + a) * BS + tid]; };
        T out[D][D][D];
#pragma unroll
        for (int c = 0; c < D; ++c)
#pragma unroll
            for (int b = 0; b < D; ++b)
#pragma unroll
                for (int a = 0; a < D; ++a) out[c][b][a] = T(0);
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
                T C0[D][QH], C1[D][QH], C2[D][QH];  // [c][qx - h0]
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
#pragma unroll
                for (int k = 0; k < QH; ++k) {
                    const int j = qy * Q + h0 + k;  // column = stream stage
                    const int st = j % S;
                    wait_stage(&qbw[st], (j / S) & 1, A.err, wlim, ok, q_waited, j + 1);
                    const T *qc = qsw + st * STAGE + lane;
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
                        const T *qq = qc + qz * (NC * 32);
                        vx[qz] = vy[qz] = vz[qz] = vu[qz] = T(0);
                        if (HK) {
                            const T d0 = qq[0], d1 = qq[32], d2 = qq[64], d3 = qq[96], d4 = qq[128], d5 = qq[160];
                            vx[qz] = d0 * gx + d1 * gy + d2 * gz;
                            vy[qz] = d1 * gx + d3 * gy + d4 * gz;
                            vz[qz] = d2 * gx + d4 * gy + d5 * gz;
                        }
                        if (HM) vu[qz] = qq[(HK ? 6 : 0) * 32] * ui;
                    }
                    __syncwarp();
                    if (lane == 0 && ok && j + S < COLS) {
                        fence_proxy_async();
                        mbar_arrive_expect_tx(&qbw[st], QBYTES);
                        bulk_g2s(qsw + st * STAGE, qdw + (int64_t)(j + S) * STAGE, QBYTES, &qbw[st]);
                        q_issued = j + S + 1;
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
                }
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
        // the element result replaces the element values in the thread's own column
#pragma unroll
        for (int c = 0; c < D; ++c)
#pragma unroll
            for (int b = 0; b < D; ++b)
#pragma unroll
                for (int a = 0; a < D; ++a) xs[((c * D + b) * D + a) * BS + tid] = out[c][b][a];
        // after a timeout: wait out the copies still in flight
        if (!ok && lane == 0) drain_stages(qbw, S, q_waited, q_issued);
    }  // wvalid
    // E^T: the chunk's DOF sums.  The lists are staged where the rings were; a
    // CTA in which a wait timed out (error word set) stores nothing, so that no
    // copy that is still late can land in the staged lists.
    if (__syncthreads_or(!ok)) return;
    ChunkStage st = chunk_stage_at(A.L, hex_smem);
    chunk_stage_lists<BS>(A.L, blockIdx.x, st);
    __syncthreads();
    chunk_sums<T, BS>(A.L, st, xs, A.ess, A.x, A.y, A.accumulate, A.constrained, 0);
}

// Jacobi diagonal: element diagonal sum_q g_i^T D_q g_i (+ m_q phi_i^2), one
// thread per element of a chunk of BS elements, summed per DOF by the chunk
// scatter (1 on the essential DOFs of a constrained call).
template <int P, int OPK, int BS>
__global__ void __launch_bounds__(BS) hex_diag_kernel(const HexApply<double> A) {
    constexpr int D = P + 1, Q = P + 1, NL = D * D * D, NC = NComp<OPK>::v;
    constexpr bool HM = (OPK & 1) != 0, HK = (OPK & 2) != 0;
    using TB = Tab<double>;
    extern __shared__ __align__(128) unsigned char hex_smem[];
    double *ys = reinterpret_cast<double *>(hex_smem);  // [NL][BS]
    const int tid = threadIdx.x;
    const int64_t e = (int64_t)blockIdx.x * BS + tid;
    const int64_t E = A.E;
    double out[D][D][D];
#pragma unroll
    for (int c = 0; c < D; ++c)
#pragma unroll
        for (int b = 0; b < D; ++b)
#pragma unroll
            for (int a = 0; a < D; ++a) out[c][b][a] = 0.0;
    if (e < E && __ldg(A.dofs + e) >= 0) {
        for (int qy = 0; qy < Q; ++qy)
            for (int qx = 0; qx < Q; ++qx)
                for (int qz = 0; qz < Q; ++qz) {
                    double d[7];
#pragma unroll
                    for (int k = 0; k < NC; ++k) d[k] = __ldg(A.qd + hex_qd_index<P, OPK>(e, qy * Q + qx, qz, k));
#pragma unroll
                    for (int c = 0; c < D; ++c)
#pragma unroll
                        for (int b = 0; b < D; ++b)
#pragma unroll
                            for (int a = 0; a < D; ++a) {
                                const double Bx = TB::B(P, qx, a), By = TB::B(P, qy, b), Bz = TB::B(P, qz, c);
                                double s = 0.0;
                                if (HK) {
                                    const double gx = TB::G(P, qx, a) * By * Bz;
                                    const double gy = Bx * TB::G(P, qy, b) * Bz;
                                    const double gz = Bx * By * TB::G(P, qz, c);
                                    s = d[0] * gx * gx + d[3] * gy * gy + d[5] * gz * gz +
                                        2.0 * (d[1] * gx * gy + d[2] * gx * gz + d[4] * gy * gz);
                                }
                                if (HM) {
                                    const double ph = Bx * By * Bz;
                                    s += d[HK ? 6 : 0] * ph * ph;
                                }
                                out[c][b][a] += s;
                            }
                }
    }
#pragma unroll
    for (int c = 0; c < D; ++c)
#pragma unroll
        for (int b = 0; b < D; ++b)
#pragma unroll
            for (int a = 0; a < D; ++a) ys[((c * D + b) * D + a) * BS + tid] = out[c][b][a];
    ChunkStage st = chunk_stage_at(A.L, hex_smem + sizeof(double) * NL * BS);
    chunk_stage_lists<BS>(A.L, blockIdx.x, st);
    __syncthreads();
    chunk_sums<double, BS>(A.L, st, ys, A.ess, nullptr, A.y, 0, A.constrained, 1);
}

// Quadrature-data setup of the unstructured mesh: one thread per (element,
// point).  Sorted element s is the caller's element eid[s]; its vertices are
// conn[eid*8 .. +8] in HexQ1 order; kappa_q / rho_q are indexed by the
// caller's element and the tensor point (qz, qy, qx).
struct HexSetup {
    int64_t E;              // padded element count
    const int32_t *eid;     // [E] sorted -> caller element, -1 for padding
    const uint32_t *conn;   // [E][8]
    const double *coords;   // [n_nodes][3]
    const double *kappa_q, *rho_q;
    double kappa_c, rho_c, c_m, c_k;
    double gx[4], gw[4];
    int *err;
};

template <int P, int OPK, typename T>
__global__ void hex_setup_kernel(const HexSetup S, T *__restrict__ qd) {
    constexpr int Q = P + 1, Q3 = Q * Q * Q, NC = NComp<OPK>::v;
    constexpr bool HM = (OPK & 1) != 0, HK = (OPK & 2) != 0;
    const int64_t total = S.E * Q3;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = t / Q3;
        const int q = (int)(t % Q3);  // tensor point index (qz, qy, qx), qx fastest
        const int qx = q % Q, qy = (q / Q) % Q, qz = q / (Q * Q);
        const int64_t e = S.eid[s];
        if (e < 0) {  // padding element: zero data
            if (HK)
                for (int k = 0; k < 6; ++k) qd[hex_qd_index<P, OPK>(s, qy * Q + qx, qz, k)] = (T)0;
            if (HM) qd[hex_qd_index<P, OPK>(s, qy * Q + qx, qz, HK ? 6 : 0)] = (T)0;
            continue;
        }
        double xv[8][3];
        for (int k = 0; k < 8; ++k) {
            const int64_t v = S.conn[e * 8 + k];
            xv[k][0] = S.coords[3 * v];
            xv[k][1] = S.coords[3 * v + 1];
            xv[k][2] = S.coords[3 * v + 2];
        }
        const double xi[3] = {S.gx[qx], S.gx[qy], S.gx[qz]};
        const double w = S.gw[qx] * S.gw[qy] * S.gw[qz];
        const double kap = S.kappa_q ? S.kappa_q[e * Q3 + q] : S.kappa_c;
        const double rho = S.rho_q ? S.rho_q[e * Q3 + q] : S.rho_c;
        double D[6], m;
        if (!hex_point_qdata(xv, xi, w, kap, S.c_k, rho, S.c_m, D, m) && S.err) atomicOr(S.err, FG_DERR_BOUNDS);
        if (HK)
            for (int k = 0; k < 6; ++k) qd[hex_qd_index<P, OPK>(s, qy * Q + qx, qz, k)] = (T)D[k];
        if (HM) qd[hex_qd_index<P, OPK>(s, qy * Q + qx, qz, HK ? 6 : 0)] = (T)m;
        (void)NC;
    }
}

}  // namespace fg
