// tet_kernels.cuh -- partial-assembly operator on unstructured tetrahedra
// (TetP1 / TetP2), the element path of crates/assembly/src/partial.rs on Tet4.
//
// Data layout (element-major structure of arrays, one coalesced load per
// component across a warp of consecutive elements):
//   dofs [nl][E]  int32 element-to-DOF map (first 4 = vertex nodes)
//   G    [6][E]   |det J| J^-1 J^-T (symmetric: xx xy xz yy yz zz), constant
//                 per element (affine map)
//   sk   [nq][E]  w_q kappa_q c_k          (diffusion)
//   sm   [nq][E]  w_q |det J| rho_q c_m    (mass)
//   Ye   [E][nl]  element-local results (scratch; element-major so that the
//                 slots of one DOF, which come from nearby elements, share sectors)
// Per quadrature point the reference computes grad_phys = J^-T grad_ref and
// y_i += w |det J| kappa (grad u . grad phi_i); with the affine map this is
// y_i += (w kappa) grad_ref phi_i . G grad_ref u, which the apply evaluates.
//
// Scatter without float atomics: the transpose of the element-to-DOF map is a
// CSR list per DOF of element-local slots (e*nl + i) in increasing (e, i); one
// thread per DOF sums its slots in that order (deterministic).
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
    TetRule R;
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

// Ye[e][i] = (A_e x_e)_i (diag = 0) or (A_e)_ii (diag = 1), one thread per element
template <int NL, int MQ>
__global__ void __launch_bounds__(128) tet_apply_kernel(TetArgs A, const __grid_constant__ TetTab<NL, MQ> R,
                                                        const double *__restrict__ x, double *__restrict__ Ye,
                                                        int constrained, int diag) {
    const int64_t E = A.E;
    const int nq = A.R.nq;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        double xe[NL], ye[NL];
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
        double *dst = Ye + e * NL;
#pragma unroll
        for (int i = 0; i < NL; ++i) dst[i] = ye[i];
    }
}

// y_d (+)= sum of the element-local slots of DOF d in (e, i) order; on
// essential DOFs of a constrained call the identity row: y_d (+)= x_d (apply)
// or 1 (diagonal, x null)
__global__ void tet_scatter_kernel(TetArgs A, const int64_t *__restrict__ offs, const int32_t *__restrict__ slots,
                                   const double *__restrict__ Ye, const double *__restrict__ x,
                                   double *__restrict__ y, int accumulate, int constrained) {
    for (int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d < A.N; d += (int64_t)gridDim.x * blockDim.x) {
        double s;
        if (constrained && A.ess && A.ess[d]) {
            s = x ? x[d] : 1.0;
        } else {
            s = 0.0;
            for (int64_t k = offs[d]; k < offs[d + 1]; ++k) s += Ye[slots[k]];
        }
        y[d] = accumulate ? y[d] + s : s;
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
