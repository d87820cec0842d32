// tet_kernels.cuh -- partial-assembly operator on unstructured tetrahedra
// (TetP1 / TetP2 / TetP3), the element path of crates/assembly/src/partial.rs
// on Tet4.
//
// Per quadrature point the reference computes grad_phys = J^-T grad_ref and
// y_i += w |det J| kappa (grad u . grad phi_i); with the affine map this is
// y_i += (w kappa) grad_ref phi_i . G grad_ref u, G = |det J| J^-1 J^-T
// (constant per element), which the apply evaluates.
//
// Moment form (diffusion, P1 and P2).  The reference gradients of P1/P2 are
// affine in xi: grad_ref u(xi) = g0 + H xi (H symmetric, the Hessian of u; 0
// for P1).  With s_q = w_q kappa_q c_k the quadrature sum is then exactly
//   y_i = a_i . G M0 + sum_k B_i[:,k] . G M_k,   grad_ref phi_i = a_i + B_i xi,
//   M0 = S00 g0 + H s1,   M_k = s1_k g0 + H S2[:,k],
// with the per-element moments S00 = sum s_q, s1 = sum s_q xi_q and
// S2 = sum s_q xi_q xi_q^T (10 numbers, P1: S00 only), so the apply reads 10
// numbers per element instead of nq point scalars and does ~160 FMAs instead
// of ~70 nq.  The mass term, P3 and the diagonal use the point form.
//
// Layout (element-major structure of arrays in a locality order of the
// elements, one coalesced load per component across a warp):
//   G    [6][E]    |det J| J^-1 J^-T (xx xy xz yy yz zz)
//   Sm   [10][E]   diffusion moments (S00, s1, S2 as xx xy xz yy yz zz); P1: [6][E] S00 G
//   sk   [nq][E]   w_q kappa_q c_k          (diffusion, point form)
//   sm   [nq][E]   w_q |det J| rho_q c_m    (mass)
//   edof [nl][E]   int32 element-to-DOF map
//   emsk [E]       uint32 bit i set: local DOF i is essential
//
// Scatter without float atomics and without an element-result array in HBM:
// the elements, sorted along a Morton curve of their centroids, form chunks
// of CE elements, one CTA each.  A chunk computes its element results into
// shared memory and sums, per DOF of its list, the element-local slots of
// that DOF in increasing (local index, element) order.  A DOF whose elements all lie in the chunk is
// stored directly; a DOF shared with other chunks gets one partial sum per
// chunk, and chunk_shared_kernel adds the partials of each such DOF in
// increasing chunk order (chunk_plan.h, chunk_scatter.cuh).  The result is
// deterministic.
#pragma once
#include "chunk_scatter.cuh"
#include "fg_common.cuh"

namespace fg {

constexpr int TET_MAXQ = 35;  // Grundmann-Moller s = 3

struct TetRule {
    int nq;
    const double *phi;   // [nq][nl] basis values at the points
    const double *grad;  // [nq][nl][3] reference gradients
};

struct TetArgs {
    int64_t E, N;
    int kind;                  // bit 1 mass, bit 2 diffusion
    const int32_t *dofs;       // [nl][E] caller's element order
    const double *G;           // [6][E]
    const double *sk, *sm;     // [nq][E]
    const uint8_t *ess;        // [N] or null
    TetRule R;
};

// Chunked apply: element data in the chunk order, chunk DOF lists.
struct TetChunk {
    int64_t E, N;
    int CE;                      // elements per chunk
    const double *G, *Sm;        // [6][E], [10][E] (P1: [6][E] S00 G)
    const double *sk, *sm;       // [nq][E]
    const int32_t *edof;         // [nl][E]
    const uint32_t *emsk;        // [E] essential local DOFs (bit i), null if no essential list
    const uint8_t *ess;          // [N] or null
    ChunkLists L;
};

// one thread per element: geometry and the per-point scalars
__global__ void tet_setup_kernel(TetArgs A, int nl, const double *__restrict__ coords,
                                 const double *__restrict__ qw, const double *__restrict__ kappa_q, double kappa_c,
                                 const double *__restrict__ rho_q, double rho_c, double c_m, double c_k,
                                 double *G, double *sk, double *sm, int *err) {
    const int64_t E = A.E;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        const double *x0 = coords + 3 * (int64_t)A.dofs[e];
        double J[3][3];
        for (int c = 0; c < 3; ++c) {
            const double *xc = coords + 3 * (int64_t)A.dofs[(int64_t)(c + 1) * E + e];
            for (int r = 0; r < 3; ++r) J[r][c] = xc[r] - x0[r];
        }
        const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                           J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        if (!(fabs(det) > 0.0)) atomicOr(err, FG_DERR_BOUNDS);
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
        const double ad = fabs(det);
        const int mi[6] = {0, 0, 0, 1, 1, 2}, ni[6] = {0, 1, 2, 1, 2, 2};
        for (int k = 0; k < 6; ++k) {
            const int m = mi[k], n = ni[k];
            G[(int64_t)k * E + e] = ad * (inv[m][0] * inv[n][0] + inv[m][1] * inv[n][1] + inv[m][2] * inv[n][2]);
        }
        for (int q = 0; q < A.R.nq; ++q) {
            if (A.kind & 2) sk[(int64_t)q * E + e] = qw[q] * (kappa_q ? kappa_q[e * A.R.nq + q] : kappa_c) * c_k;
            if (A.kind & 1) sm[(int64_t)q * E + e] = qw[q] * ad * (rho_q ? rho_q[e * A.R.nq + q] : rho_c) * c_m;
        }
        (void)nl;
    }
}

// Rule tables passed by value as a kernel parameter (constant bank): every
// thread of a warp reads the same entry at the same time, so the reads are
// broadcasts.  MQ = capacity in points (4 for tet_rule orders <= 2, 35 above).
template <int NL, int MQ> struct TetTab {
    double phi[MQ][NL];
    double grad[MQ][NL][3];
};

// Element results by the point form: ye = A_e xe (diag = 0) or the diagonal of
// A_e (diag = 1) for element e of the chunk order.
template <int NL, int MQ>
__device__ __forceinline__ void tet_elem_points(const TetChunk &C, int kind, int nq, const TetTab<NL, MQ> &R,
                                                int64_t e, const double (&xe)[NL], double (&ye)[NL], int diag) {
    const int64_t E = C.E;
#pragma unroll
    for (int i = 0; i < NL; ++i) ye[i] = 0.0;
    double g[6] = {0, 0, 0, 0, 0, 0};
    if (kind & 2)
#pragma unroll
        for (int k = 0; k < 6; ++k) g[k] = __ldg(C.G + (int64_t)k * E + e);
    for (int q = 0; q < nq; ++q) {
        if (kind & 2) {
            const double s = __ldg(C.sk + (int64_t)q * E + e);
            if (!diag) {
                double gu[3] = {0, 0, 0};
#pragma unroll
                for (int j = 0; j < NL; ++j)
#pragma unroll
                    for (int c = 0; c < 3; ++c) gu[c] += xe[j] * R.grad[q][j][c];
                const double v0 = s * (g[0] * gu[0] + g[1] * gu[1] + g[2] * gu[2]);
                const double v1 = s * (g[1] * gu[0] + g[3] * gu[1] + g[4] * gu[2]);
                const double v2 = s * (g[2] * gu[0] + g[4] * gu[1] + g[5] * gu[2]);
#pragma unroll
                for (int i = 0; i < NL; ++i)
                    ye[i] += R.grad[q][i][0] * v0 + R.grad[q][i][1] * v1 + R.grad[q][i][2] * v2;
            } else {
#pragma unroll
                for (int i = 0; i < NL; ++i) {
                    const double a = R.grad[q][i][0], b = R.grad[q][i][1], c = R.grad[q][i][2];
                    ye[i] += s * (g[0] * a * a + g[3] * b * b + g[5] * c * c +
                                  2.0 * (g[1] * a * b + g[2] * a * c + g[4] * b * c));
                }
            }
        }
        if (kind & 1) {
            const double m = __ldg(C.sm + (int64_t)q * E + e);
            if (!diag) {
                double u = 0.0;
#pragma unroll
                for (int j = 0; j < NL; ++j) u += R.phi[q][j] * xe[j];
                const double t = m * u;
#pragma unroll
                for (int i = 0; i < NL; ++i) ye[i] += R.phi[q][i] * t;
            } else {
#pragma unroll
                for (int i = 0; i < NL; ++i) ye[i] += m * R.phi[q][i] * R.phi[q][i];
            }
        }
    }
}

// Element diffusion result by the moment form (P1: NL = 4, P2: NL = 10).
// Gradients of the TetP1/TetP2 bases of crates/element/src/lagrange/tet.rs in
// barycentric form (l1 = 1 - x - y - z): vertex i grad (4 l_i - 1) grad l_i,
// edge (i, j) grad 4 l_i l_j; their coefficients of 1, x, y, z give g0, H and
// the a_i, B_i below.
template <int NL> struct TetMom { static constexpr int n = NL == 4 ? 6 : 16; };

// The element's moment-form data: P1 the 6 entries of S00 G, P2 G (6) and the
// 10 moments.
template <int NL>
__device__ __forceinline__ void tet_load_moments(const TetChunk &C, int64_t e, double (&md)[TetMom<NL>::n]) {
    const int64_t E = C.E;
    if constexpr (NL == 4) {
#pragma unroll
        for (int k = 0; k < 6; ++k) md[k] = __ldg(C.Sm + (int64_t)k * E + e);
    } else {
#pragma unroll
        for (int k = 0; k < 6; ++k) md[k] = __ldg(C.G + (int64_t)k * E + e);
#pragma unroll
        for (int k = 0; k < 10; ++k) md[6 + k] = __ldg(C.Sm + (int64_t)k * E + e);
    }
}

template <int NL>
__device__ __forceinline__ void tet_elem_moments(const double (&md)[TetMom<NL>::n], const double (&u)[NL],
                                                 double (&y)[NL]) {
    const double *G = md;
    auto Gv = [&](const double (&m)[3], double (&v)[3]) {
        v[0] = G[0] * m[0] + G[1] * m[1] + G[2] * m[2];
        v[1] = G[1] * m[0] + G[3] * m[1] + G[4] * m[2];
        v[2] = G[2] * m[0] + G[4] * m[1] + G[5] * m[2];
    };
    if constexpr (NL == 4) {
        const double g[3] = {u[1] - u[0], u[2] - u[0], u[3] - u[0]};
        double v[3];
        Gv(g, v);  // G holds S00 G
        y[0] = -(v[0] + v[1] + v[2]);
        y[1] = v[0];
        y[2] = v[1];
        y[3] = v[2];
    } else {
        const double *S = md + 6;
        // g0 and the Hessian H (xx yy zz xy xz yz)
        const double t0 = 3.0 * u[0], f0 = 4.0 * u[0];
        const double g0[3] = {4.0 * u[4] - t0 - u[1], 4.0 * u[5] - t0 - u[2], 4.0 * u[6] - t0 - u[3]};
        const double hxx = 4.0 * (u[0] + u[1]) - 8.0 * u[4];
        const double hyy = 4.0 * (u[0] + u[2]) - 8.0 * u[5];
        const double hzz = 4.0 * (u[0] + u[3]) - 8.0 * u[6];
        const double hxy = f0 + 4.0 * (u[7] - u[4] - u[5]);
        const double hxz = f0 + 4.0 * (u[8] - u[4] - u[6]);
        const double hyz = f0 + 4.0 * (u[9] - u[5] - u[6]);
        auto Hv = [&](double a, double b, double c, double (&v)[3]) {
            v[0] = hxx * a + hxy * b + hxz * c;
            v[1] = hxy * a + hyy * b + hyz * c;
            v[2] = hxz * a + hyz * b + hzz * c;
        };
        // S = (S00, s1x, s1y, s1z, S2xx, S2xy, S2xz, S2yy, S2yz, S2zz)
        double m[3], v0[3], w[3][3];  // w[k] = G M_{k+1}
        Hv(S[1], S[2], S[3], m);
#pragma unroll
        for (int c = 0; c < 3; ++c) m[c] += S[0] * g0[c];
        Gv(m, v0);
        const double s2c[3][3] = {{S[4], S[5], S[6]}, {S[5], S[7], S[8]}, {S[6], S[8], S[9]}};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            Hv(s2c[k][0], s2c[k][1], s2c[k][2], m);
#pragma unroll
            for (int c = 0; c < 3; ++c) m[c] += S[1 + k] * g0[c];
            Gv(m, w[k]);
        }
        // W[c][k] = w[k][c]; diagonal and symmetric off-diagonal sums
        const double d0 = w[0][0], d1 = w[1][1], d2 = w[2][2];
        const double o01 = w[1][0] + w[0][1], o02 = w[2][0] + w[0][2], o12 = w[2][1] + w[1][2];
        y[0] = -3.0 * (v0[0] + v0[1] + v0[2]) + 4.0 * (d0 + d1 + d2 + o01 + o02 + o12);
        y[1] = 4.0 * d0 - v0[0];
        y[2] = 4.0 * d1 - v0[1];
        y[3] = 4.0 * d2 - v0[2];
        y[4] = 4.0 * (v0[0] - 2.0 * d0 - o01 - o02);
        y[5] = 4.0 * (v0[1] - 2.0 * d1 - o01 - o12);
        y[6] = 4.0 * (v0[2] - 2.0 * d2 - o02 - o12);
        y[7] = 4.0 * o01;
        y[8] = 4.0 * o02;
        y[9] = 4.0 * o12;
    }
}

// Shared-memory plan of a chunk (bytes): element results, then the chunk's
// lists.
__host__ __device__ inline size_t tet_chunk_smem(int NL, int CE, int max_nu) {
    return sizeof(double) * (size_t)NL * CE + chunk_list_smem(NL, CE, max_nu);
}

// One CTA (BT threads) per chunk.  First the chunk's DOF list (ids, partial
// ids, slot offsets relative to the chunk) and local slots are staged in
// shared memory and the element results are computed into shared memory, the
// element gathering its x values through the element map: no wait separates
// the two, so all their loads are in flight together.  After the barrier each
// DOF's slots are summed from shared memory.  MOM: diffusion-only apply by the
// moment form.  On essential DOFs of a constrained call the identity row:
// y_d (+)= x_d (apply) or 1 (diagonal).
template <int NL, int MQ, bool MOM, int BT>
__global__ void __launch_bounds__(BT, MOM ? (BT == 512 ? 2 : 3) : 1) tet_chunk_kernel(const TetChunk C, int kind, int nq,
                                                                  const __grid_constant__ TetTab<NL, MQ> R,
                                                                  const double *__restrict__ x,
                                                                  double *__restrict__ y, int accumulate,
                                                                  int constrained, int diag) {
    extern __shared__ __align__(16) unsigned char tsm_raw[];
    const int CE = C.CE;
    double *ys = reinterpret_cast<double *>(tsm_raw);  // [NL][CE] element results
    ChunkStage S = chunk_stage_at(C.L, tsm_raw + sizeof(double) * NL * CE);
    const int c = blockIdx.x;
    const int64_t e0 = (int64_t)c * CE;
    const int ne = (int)(C.E - e0 < CE ? C.E - e0 : CE);
    chunk_stage_lists<BT>(C.L, c, S);
    const bool mask = constrained && C.emsk;
    for (int el = threadIdx.x; el < ne; el += BT) {
        const int64_t e = e0 + el;
        double xe[NL], ye[NL];
        double md[MOM ? TetMom<NL>::n : 1];
        if constexpr (MOM) tet_load_moments<NL>(C, e, md);  // issued before the dependent x gathers
        const uint32_t m = mask ? __ldg(C.emsk + e) : 0u;
#pragma unroll
        for (int i = 0; i < NL; ++i) {
            xe[i] = 0.0;
            if (!diag) {
                const double v = __ldg(x + __ldg(C.edof + (int64_t)i * C.E + e));
                xe[i] = ((m >> i) & 1u) ? 0.0 : v;
            }
        }
        if constexpr (MOM) tet_elem_moments<NL>(md, xe, ye);
        else tet_elem_points<NL, MQ>(C, kind, nq, R, e, xe, ye, diag);
#pragma unroll
        for (int i = 0; i < NL; ++i) ys[i * CE + el] = ye[i];
    }
    __syncthreads();
    chunk_sums<double, BT>(C.L, S, ys, C.ess, x, y, accumulate, constrained, diag);
}

// Reorder the per-element data into the chunk order and form the diffusion
// moments from the point scalars (nmom = 10 for P2; 6 for P1, where the only
// moment S00 is stored multiplied into G; 0 otherwise).
__global__ void tet_permute_kernel(int64_t E, int nq, int kind, int nmom, const int32_t *__restrict__ perm,
                                   const double *__restrict__ qp, const double *__restrict__ G,
                                   const double *__restrict__ sk, const double *__restrict__ sm, double *Gp,
                                   double *skp, double *smp, double *Sm) {
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < E; n += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = perm[n];
        for (int k = 0; k < 6; ++k) Gp[(int64_t)k * E + n] = G[(int64_t)k * E + e];
        double mo[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int q = 0; q < nq; ++q) {
            if (kind & 2) {
                const double s = sk[(int64_t)q * E + e];
                skp[(int64_t)q * E + n] = s;
                const double a = qp[3 * q], b = qp[3 * q + 1], c = qp[3 * q + 2];
                mo[0] += s;
                mo[1] += s * a;
                mo[2] += s * b;
                mo[3] += s * c;
                mo[4] += s * a * a;
                mo[5] += s * a * b;
                mo[6] += s * a * c;
                mo[7] += s * b * b;
                mo[8] += s * b * c;
                mo[9] += s * c * c;
            }
            if (kind & 1) smp[(int64_t)q * E + n] = sm[(int64_t)q * E + e];
        }
        if (nmom == 6)  // P1: S00 G
            for (int k = 0; k < 6; ++k) Sm[(int64_t)k * E + n] = mo[0] * G[(int64_t)k * E + e];
        else
            for (int k = 0; k < nmom; ++k) Sm[(int64_t)k * E + n] = mo[k];
    }
}

// Gauss points in physical space: xyz[e][q][3] = x_0 + J xi_q
__global__ void tet_qp_coords_kernel(TetArgs A, const double *__restrict__ coords, const double *__restrict__ qp,
                                     double *__restrict__ xyz) {
    const int nq = A.R.nq;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < A.E * nq; t += (int64_t)gridDim.x * blockDim.x) {
        const int q = (int)(t % nq);
        const int64_t e = t / nq;
        const double *x0 = coords + 3 * (int64_t)A.dofs[e];
        const double *xi = qp + 3 * q;
        for (int r = 0; r < 3; ++r) {
            double s = x0[r];
            for (int c = 0; c < 3; ++c) {
                const double *xc = coords + 3 * (int64_t)A.dofs[(int64_t)(c + 1) * A.E + e];
                s += (xc[r] - x0[r]) * xi[c];
            }
            xyz[3 * t + r] = s;
        }
    }
}

}  // namespace fg
