// tet_kernels.cuh -- partial-assembly operator on unstructured tetrahedra
// (TetP1 / TetP2), the element path of crates/assembly/src/partial.rs on Tet4.
//
// Data layout (elements sorted by colour, element-major structure of arrays,
// one coalesced load per component across a warp of consecutive elements):
//   dofs [nl][E]  int32 element-to-DOF map (first 4 = vertex nodes)
//   G    [6][E]   |det J| J^-1 J^-T (symmetric: xx xy xz yy yz zz), constant
//                 per element (affine map)
//   sk   [nq][E]  w_q kappa_q c_k          (diffusion)
//   sm   [nq][E]  w_q |det J| rho_q c_m    (mass)
//   eid  [E]      the caller's index of each sorted element
// Per quadrature point the reference computes grad_phys = J^-T grad_ref and
// y_i += w |det J| kappa (grad u . grad phi_i); with the affine map this is
// y_i += (w kappa) grad_ref phi_i . G grad_ref u, which the apply evaluates.
//
// Scatter without float atomics: the elements are coloured so that no two
// elements of a colour share a DOF.  One cooperative launch walks the colours
// in order with a grid barrier between them, and each element adds its result
// into y directly: every DOF receives its contributions in colour order, the
// same sums every run, with no element-result round trip through HBM.
#pragma once
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
    const int32_t *dofs;       // [nl][E]
    const double *G;           // [6][E]
    const double *sk, *sm;     // [nq][E]
    const uint8_t *ess;        // [N] or null
    const int32_t *eid;        // [E] sorted -> caller element
    TetRule R;
};

// Colour ranges of the sorted elements (at most 64 colours).
struct TetColours {
    int64_t start[65];
    int ncol;
};

// one thread per element: geometry and the per-point scalars
__global__ void tet_setup_kernel(TetArgs A, int nl, const double *__restrict__ coords,
                                 const double *__restrict__ qw, const double *__restrict__ kappa_q, double kappa_c,
                                 const double *__restrict__ rho_q, double rho_c, double c_m, double c_k,
                                 double *G, double *sk, double *sm, int *err) {
    const int64_t E = A.E;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ec = A.eid[e];  // the caller's element (coefficient tables)
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
            if (A.kind & 2) sk[(int64_t)q * E + e] = qw[q] * (kappa_q ? kappa_q[ec * A.R.nq + q] : kappa_c) * c_k;
            if (A.kind & 1) sm[(int64_t)q * E + e] = qw[q] * ad * (rho_q ? rho_q[ec * A.R.nq + q] : rho_c) * c_m;
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

// ye = (A_e x_e) (diag = 0) or the element diagonal (diag = 1) of element e
template <int NL, int MQ>
__device__ __forceinline__ void tet_element(const TetArgs &A, const TetTab<NL, MQ> &R, const double *__restrict__ x,
                                            int64_t e, int constrained, int diag, double (&ye)[NL]) {
    const int64_t E = A.E;
    const int nq = A.R.nq;
    double xe[NL];
#pragma unroll
    for (int i = 0; i < NL; ++i) {
        ye[i] = 0.0;
        xe[i] = 0.0;
        if (!diag) {
            const int32_t d = __ldg(A.dofs + (int64_t)i * E + e);
            xe[i] = (constrained && A.ess && A.ess[d]) ? 0.0 : __ldg(x + d);
        }
    }
    double g[6] = {0, 0, 0, 0, 0, 0};
    if (A.kind & 2)
#pragma unroll
        for (int k = 0; k < 6; ++k) g[k] = __ldg(A.G + (int64_t)k * E + e);
    for (int q = 0; q < nq; ++q) {
        if (A.kind & 2) {
            const double s = __ldg(A.sk + (int64_t)q * E + e);
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
        if (A.kind & 1) {
            const double m = __ldg(A.sm + (int64_t)q * E + e);
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

// The whole apply in one cooperative launch: y = (accumulate ? y : 0) + the
// identity rows of the essential DOFs of a constrained call (x, or 1 for the
// diagonal); then the colours in order, a grid barrier after each, every
// element adding its result into its non-essential DOFs.  y is read at L2
// (__ldcg): another SM may have written the DOF in an earlier colour.
template <int NL, int MQ>
__global__ void __launch_bounds__(128) tet_apply_coloured_kernel(TetArgs A, const __grid_constant__ TetTab<NL, MQ> R,
                                                                 const __grid_constant__ TetColours C,
                                                                 const double *__restrict__ x, double *y,
                                                                 int accumulate, int constrained, int diag,
                                                                 unsigned *bar, int *err) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int64_t d = t0; d < A.N; d += stride) {
        double v = accumulate ? y[d] : 0.0;
        if (constrained && A.ess && A.ess[d]) v += diag ? 1.0 : x[d];
        y[d] = v;
    }
    bool ok = true;
    for (int c = 0; c < C.ncol; ++c) {
        grid_barrier(bar, err, ok);
        for (int64_t e = C.start[c] + t0; e < C.start[c + 1]; e += stride) {
            double ye[NL];
            tet_element<NL, MQ>(A, R, x, e, constrained, diag, ye);
#pragma unroll
            for (int i = 0; i < NL; ++i) {
                const int32_t d = __ldg(A.dofs + (int64_t)i * A.E + e);
                if (!(constrained && A.ess && A.ess[d])) y[d] = __ldcg(y + d) + ye[i];
            }
        }
    }
}

// Gauss points in physical space: xyz[e][q][3] = x_0 + J xi_q
__global__ void tet_qp_coords_kernel(TetArgs A, const double *__restrict__ coords, const double *__restrict__ qp,
                                     double *__restrict__ xyz) {
    const int nq = A.R.nq;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < A.E * nq; t += (int64_t)gridDim.x * blockDim.x) {
        const int q = (int)(t % nq);
        const int64_t e = t / nq;  // sorted element; the output is in the caller's element order
        const double *x0 = coords + 3 * (int64_t)A.dofs[e];
        const double *xi = qp + 3 * q;
        for (int r = 0; r < 3; ++r) {
            double s = x0[r];
            for (int c = 0; c < 3; ++c) {
                const double *xc = coords + 3 * (int64_t)A.dofs[(int64_t)(c + 1) * A.E + e];
                s += (xc[r] - x0[r]) * xi[c];
            }
            xyz[3 * ((int64_t)A.eid[e] * nq + q) + r] = s;
        }
    }
}

}  // namespace fg
