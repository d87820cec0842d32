/*
 * femoracle.h -- CPU oracle for the partial-assembly (PA) operator + PCG path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA
 * product path is compared against, and the timed CPU baseline ("port" of the
 * reference algorithm).  Nothing in the product library links or calls it.
 *
 * It restates, in plain C, the algorithms of the fem-rs reference
 * (javagg/fem-rs, a Rust workspace that cannot be compiled here: no Rust
 * toolchain, and its `linger` / `reed` dependencies are not vendored):
 *
 *   - PA mass / diffusion apply: crates/assembly/src/partial.rs:85-130,154-208
 *     (element loop, per-quadrature-point basis evaluation, dense
 *     sum over local DOFs, scatter y[g] += y_e), extended to Hex8 with the
 *     isoparametric Jacobian of crates/assembly/src/assembler.rs:96-143.
 *   - Hex Q1 basis and node order: crates/element/src/lagrange/hex.rs:13-66.
 *   - 1-D equispaced Lagrange conventions: crates/element/src/lagrange/quad.rs:92-105
 *     (Q2 nodes {-1,0,1}), crates/element/src/lagrange/seg.rs:119-121 (P3 nodes).
 *     Q2/Q3 hexahedra do not exist in the reference; the tensor-product
 *     equispaced Lagrange element used here is this project's definition.
 *   - Gauss-Legendre rules: crates/element/src/quadrature.rs:12-32,405-419.
 *   - Mesh numbering and boundary tags: crates/mesh/src/simplex.rs:591-679
 *     (nid = k*np^2 + j*np + i; tags 1..6 = z0,z1,y0,y1,x0,x1).
 *   - Dirichlet row/column elimination: crates/space/src/constraints.rs:31-42,
 *     crates/linalg/src/csr.rs:297-312 (with x0 = 0 and homogeneous data the
 *     row-zeroed system has the same iterates as the symmetric eliminated one).
 *   - PCG-Jacobi: crates/parallel/src/par_solver.rs:262-342 (inverse diagonal
 *     1/d if |d| > 1e-30 else 1; stop when ||r||/||b|| < rtol every iteration).
 *   - Operator CG: crates/solver/src/lib.rs:198-278.
 *   - Reference Chebyshev smoother (compat only): crates/amg/src/lib.rs:53-103;
 *     power iteration: crates/amg/src/lib.rs:108-123.
 *   - Textbook Chebyshev on D^-1 A (Saad, Iterative Methods for Sparse Linear
 *     Systems, 2nd ed., Alg. 12.1): the reference's recurrence diverges with
 *     correct bounds, so the solver path uses the textbook one.
 *   - Domain source: crates/assembly/src/standard/source.rs:39-50 with the
 *     quadrature order 2p+1 of examples/mfem_ex1_poisson.rs:81,87.
 *   - SDIRK-2 heat stage systems: examples/mfem_ex10_heat_equation.rs:201-250,
 *     gamma = 1 - 1/sqrt(2) (crates/solver/src/ode.rs:441).
 *
 * Parity pins: the reference ships no golden vectors for this path.  The
 * oracle is pinned against the reference's own known-answer tests, restated
 * in tests/test_oracle_kat.py (PA vs assembled <= 1e-11, K*1 = 0 <= 1e-12,
 * linearity <= 1e-13, 1'M1 = |Omega|, Q1 partition of unity / Kronecker,
 * Gauss weight sums, ex1 L2 error and rate bounds).
 */
#ifndef FEMORACLE_H
#define FEMORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Structured hexahedral box mesh: nx*ny*nz elements, trilinear geometry
 * from the (nx+1)(ny+1)(nz+1) vertex coordinates (lexicographic, i fastest,
 * 3 doubles each; NULL = uniform unit cube).  Order-p DOFs live on the
 * lexicographic (nx*p+1)(ny*p+1)(nz*p+1) grid. */
typedef struct {
    int nx, ny, nz;
    int p;          /* polynomial order 1..3 */
    int nq;         /* 1-D Gauss points 1..4 */
    const double *vcoord;
} or_mesh;

/* Operator kinds (bit flags): 1 = mass, 2 = diffusion, 3 = c_m*M + c_k*K. */
enum { OR_MASS = 1, OR_DIFF = 2, OR_MASS_DIFF = 3 };

void   or_gauss_legendre(int n, double *x, double *w);
int    or_hex_rule_points(int order);
void   or_lagrange1d(int p, double xi, double *phi, double *dphi);
void   or_hexq1_basis(const double xi[3], double phi[8], double grad[24]);
int64_t or_ndofs(const or_mesh *m);
void   or_elem_dofs(const or_mesh *m, int64_t e, int64_t *dofs);
void   or_unit_cube_vertices(int nx, int ny, int nz, double *vc);

/* y (+)= A x with the reference algorithm.  kappa_q / rho_q: per-quadrature
 * point coefficients [E][qz][qy][qx] or NULL for the constants.  A = c_m*M +
 * c_k*K restricted by `kind`.  No boundary conditions. */
int or_pa_apply(const or_mesh *m, int kind, double c_m, double c_k,
                const double *kappa_q, double kappa_c,
                const double *rho_q, double rho_c,
                const double *x, double *y, int accumulate, int nthreads);

/* Element matrix (D^3 x D^3, row-major, lexicographic local order). */
int or_element_matrix(const or_mesh *m, int64_t e, int kind, double c_m, double c_k,
                      const double *kappa_q, double kappa_c,
                      const double *rho_q, double rho_c, double *Ke);

/* Essential-DOF mask from boundary tags (bit t-1 set = tag t Dirichlet). */
void or_ess_mask(const or_mesh *m, int tag_bits, uint8_t *mask);

/* Constrained operator: y = A x~ with x~ = x on free DOFs, 0 on essential
 * DOFs; y[ess] = x[ess]. */
int or_apply_constrained(const or_mesh *m, int kind, double c_m, double c_k,
                         const double *kappa_q, double kappa_c,
                         const double *rho_q, double rho_c,
                         const uint8_t *ess, const double *x, double *y, int nthreads);

/* Diagonal of the constrained operator (1 on essential DOFs). */
int or_diagonal(const or_mesh *m, int kind, double c_m, double c_k,
                const double *kappa_q, double kappa_c,
                const double *rho_q, double rho_c,
                const uint8_t *ess, double *d, int nthreads);

/* b_i = sum_q w |detJ| f(x_q) phi_i; f_kind 1: 3 pi^2 sin(pi x) sin(pi y) sin(pi z).
 * Quadrature with nq points per direction.  Essential entries set to 0. */
int or_source(const or_mesh *m, int f_kind, int nq, const uint8_t *ess, double *b);

/* L2 error against u = sin(pi x) sin(pi y) sin(pi z) with nq points. */
double or_l2_error_sin(const or_mesh *m, int nq, const double *u);

/* Row-sum lumped mass (partial.rs:222-248); rho_q [E][q^3] or NULL for rho_c. */
int or_lumped_mass(const or_mesh *m, const double *rho_q, double rho_c, int nq, double *diag);

typedef struct {
    int precond;        /* 0 none (operator CG), 1 Jacobi, 2 Chebyshev(D^-1 A) */
    int cheb_degree;    /* Chebyshev sweeps (first sweep from zero needs no apply) */
    double lmin, lmax;  /* Chebyshev bounds on D^-1 A */
    double rtol, atol;
    int max_iter;
} or_cfg;

typedef struct {
    int converged;
    int iterations;
    double final_residual;   /* ||r||/||b|| of the recurrence residual (||r|| for precond 0) */
    double true_residual;    /* ||b - A x|| / ||b|| recomputed at exit */
    int64_t applies;
} or_result;

/* PCG on the constrained operator.  x: initial guess in, solution out. */
int or_pcg(const or_mesh *m, int kind, double c_m, double c_k,
           const double *kappa_q, double kappa_c,
           const double *rho_q, double rho_c,
           const uint8_t *ess, const double *b, double *x,
           const or_cfg *cfg, or_result *res, int nthreads);

/* Power iteration on D^-1 A (constrained): returns the Rayleigh-quotient
 * estimate of lambda_max after `iters` steps from a fixed start vector. */
double or_lambda_max(const or_mesh *m, int kind, double c_m, double c_k,
                     const double *kappa_q, double kappa_c,
                     const double *rho_q, double rho_c,
                     const uint8_t *ess, int iters, int nthreads);

/* Reference compat: crates/amg/src/lib.rs:53-103 chebyshev_smooth, restated
 * over a CSR matrix, and :108-123 estimate_spectral_radius. */
void or_ref_chebyshev_smooth_csr(int64_t n, const int64_t *rowptr, const int64_t *col,
                                 const double *val, double *x, const double *b,
                                 double lmin, double lmax, int n_iter);
double or_ref_spectral_radius_csr(int64_t n, const int64_t *rowptr, const int64_t *col,
                                  const double *val, int n_iter);

#ifdef __cplusplus
}
#endif
/* ---- tetrahedra (femoracle_tet.c) ------------------------------------------
 * tet_rule(order) of quadrature.rs:259-376: returns the point count (points
 * [n][3] on the reference tet, weights summing to 1/6), -1 if cap is short. */
int or_tet_rule(int order, double *pts, double *w, int cap);
/* TetP1 / TetP2 / TetP3 basis values and reference gradients ([n][3]); returns n. */
int or_tet_basis(int p, const double xi[3], double *phi, double *grad);
/* partial.rs:85-130 / 154-208 on Tet4 elements: y (+)= A x.  coords
 * [n_nodes][3]; elem_dofs [E][4 or 10], first 4 entries = vertex nodes;
 * kappa_q / rho_q [E][nq] or NULL for the constants; kind bits 1 mass, 2
 * diffusion; ess (or NULL): identity rows and columns on marked DOFs. */
int or_tet_pa_apply(int p, int64_t n_dofs, const double *coords, int64_t n_elem, const int32_t *elem_dofs,
                    int kind, double c_m, double c_k, const double *kappa_q, double kappa_c,
                    const double *rho_q, double rho_c, int quad_order, const uint8_t *ess,
                    const double *x, double *y, int accumulate);
/* the diagonal of the same operator (1 on marked DOFs) */
int or_tet_diagonal(int p, int64_t n_dofs, const double *coords, int64_t n_elem, const int32_t *elem_dofs,
                    int kind, double c_m, double c_k, const double *kappa_q, double kappa_c,
                    const double *rho_q, double rho_c, int quad_order, const uint8_t *ess, double *d);

/* tests/poisson.rs:437-493 restated: the sin source form (ess rows zero) and
 * the L2 error against sin(pi x) sin(pi y) sin(pi z) with tet_rule(quad_order). */
int or_tet_source(int p, int64_t n_dofs, const double *coords, int64_t n_elem, const int32_t *elem_dofs,
                  int quad_order, const uint8_t *ess, double *b);
double or_tet_l2_error_sin(int p, const double *coords, int64_t n_elem, const int32_t *elem_dofs, int quad_order,
                           const double *u);

#endif
