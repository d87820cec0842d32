/*
 * femgpu.h -- C ABI of the B200 (sm_100a) partial-assembly operator + PCG
 * library (libfemgpu.so).  Plain pointers and sizes only.
 *
 * This is the drop-in boundary for fem-rs's matrix-free operator path.  Each
 * entry point names the reference interface it replaces (paths inside the
 * fem-rs workspace):
 *
 *   MatFreeOperator { apply (y += A x), apply_zero (y = A x), n_dofs }
 *       crates/assembly/src/partial.rs:45-57
 *   PAMassOperator / PADiffusionOperator ::new + ::apply
 *       crates/assembly/src/partial.rs:65-130, 138-208
 *   LinearOperator { nrows, ncols, apply (y = A x) }
 *       crates/assembly/src/backend.rs:39-46
 *   CsrMatrix::diagonal (Jacobi)          crates/linalg/src/csr.rs:245-252
 *   boundary_dofs + apply_dirichlet       crates/space/src/constraints.rs:31-120
 *   solve_cg_operator                     crates/solver/src/lib.rs:198-278
 *   solve_pcg_jacobi / par_solve_pcg_jacobi
 *       crates/solver/src/lib.rs:281-297, crates/parallel/src/par_solver.rs:262-342
 *   SolverConfig / SolveResult / SolverError
 *       crates/solver/src/lib.rs:46-142
 *   chebyshev_smooth / estimate_spectral_radius
 *       crates/amg/src/lib.rs:53-123 (textbook Chebyshev on D^-1 A instead)
 *
 * Meshes are structured hexahedral boxes (nx*ny*nz elements) with trilinear
 * geometry from arbitrary vertex positions; order p = 1..3 with p+1 Gauss
 * points per direction (hex_rule(2p+1), crates/element/src/quadrature.rs:405-419).
 * DOFs are numbered lexicographically on the (nx*p+1)(ny*p+1)(nz*p+1) grid,
 * I fastest (for p = 1 this is unit_cube_tet's node numbering,
 * crates/mesh/src/simplex.rs:608-610).
 *
 * Thread safety: calls on one handle serialise on the handle's mutex and run
 * on its CUDA stream; distinct handles are independent.
 */
#ifndef FEMGPU_H
#define FEMGPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define FG_API __attribute__((visibility("default")))
#else
#define FG_API
#endif

/* Status codes; they map 1:1 onto SolverError / FemCeedError variants
 * (crates/solver/src/lib.rs:46-54, crates/assembly/src/reed/context.rs:305-312). */
enum fg_status {
    FG_OK = 0,
    FG_CONVERGENCE_FAILED = 1, /* SolverError::ConvergenceFailed */
    FG_DIMENSION_MISMATCH = 2, /* SolverError::DimensionMismatch */
    FG_BREAKDOWN = 3,          /* SolverError::Linger("...breakdown...") */
    FG_UNSUPPORTED = 4,        /* ref_elem panic on unsupported element/order */
    FG_DEVICE_TIMEOUT = 5,     /* a bounded device-side wait ran out */
    FG_BOUNDS = 6,             /* degenerate element / bad index */
    FG_CUDA_ERROR = 7,
    FG_INVALID_ARGUMENT = 8
};

/* Operator kinds: A = c_mass*M + c_diff*K restricted to the chosen terms. */
enum fg_kind { FG_MASS = 1, FG_DIFF = 2, FG_MASS_DIFF = 3 };

/* Where the caller's vectors live. */
enum fg_mem { FG_HOST = 0, FG_DEVICE = 1 };

/* Preconditioners and precisions of fg_pcg. */
enum fg_precond { FG_PC_NONE = 0, FG_PC_JACOBI = 1, FG_PC_CHEBYSHEV = 2, FG_PC_CHEB_NN = 3 };
enum fg_precision { FG_FP64 = 0, FG_FP32_IR = 1 };

/* Quadrature-data formats (fg_op_set_qdata_format). */
enum fg_qdata_format { FG_QDATA_FULL = 0, FG_QDATA_AFFINE = 1 };

/* Boundary tags (simplex.rs:650-679 order): bit t-1 selects tag t. */
enum fg_tag {
    FG_TAG_Z0 = 1, FG_TAG_Z1 = 2, FG_TAG_Y0 = 4, FG_TAG_Y1 = 8, FG_TAG_X0 = 16, FG_TAG_X1 = 32,
    FG_TAG_ALL = 63
};

typedef struct fg_op fg_op;

typedef struct {
    int32_t nx, ny, nz;    /* elements per direction */
    const double *vcoord;  /* host or device, (nx+1)(ny+1)(nz+1)*3 vertex coordinates,
                              lexicographic i fastest; NULL = unit cube */
} fg_mesh;

typedef struct {
    double rtol;           /* converge when ||r||/||b|| < rtol (default 1e-8) */
    double atol;           /* ... or ||r|| < atol */
    int32_t max_iter;      /* default 1000 */
    int32_t print_level;   /* PrintLevel: 0 silent, 1 summary, 2 iterations */
    int32_t precond;       /* fg_precond */
    int32_t cheb_degree;   /* Chebyshev sweeps (first sweep from zero needs no apply) */
    int32_t precision;     /* fg_precision */
    int32_t power_iters;   /* power iterations on D^-1 A for lambda_max (default 20) */
    double lmax;           /* <= 0: estimate; lambda_max = lmax_safety * estimate */
    double lmin_ratio;     /* lambda_min = lambda_max / lmin_ratio (default 30) */
    double lmax_safety;    /* default 1.1 */
    double inner_rtol;     /* FP32_IR: FP32 residual reduction between FP64 reliable
                              updates (default 0.1) */
    int32_t check_interval;/* iterations between host polls of the device flag */
    int32_t nn_budget;     /* FG_PC_CHEB_NN: iterations after which an unconverged solve
                              drops the learned term and continues as plain Chebyshev-
                              preconditioned CG (0 = never); the plain solve's count */
    double nn_iter_ratio;  /* FG_PC_CHEB_NN with nn_budget > 0: the network's expected
                              ratio of learned to plain iterations (measured on
                              validation problems of its family; 0 = not known).  The
                              solver measures one plain and one learned iteration on the
                              handle (once per precision, format and degree, outside the
                              timed solve) and runs plain Chebyshev-PCG from the start
                              when ratio * learned cost >= plain cost (nn_fallback = 2) */
} fg_cfg;

typedef struct {
    int32_t converged;
    int32_t iterations;      /* PCG iterations */
    double final_residual;   /* ||r||/||b|| of the recurrence residual; ||r|| for FG_PC_NONE
                                (the operator CG's stopping rule, lib.rs:229-278) */
    double true_residual;    /* ||b - A x||/||b|| recomputed in FP64 at exit */
    int32_t status;          /* fg_status */
    int32_t outer_iterations;/* FP32_IR: FP64 reliable updates of x and the residual */
    int64_t applies;         /* operator applications */
    double lmax;             /* Chebyshev upper bound used */
    double solve_ms;         /* device time of the solve */
    int32_t nn_fallback;     /* FG_PC_CHEB_NN: 1 if the solve fell back to plain Chebyshev
                                after nn_budget iterations, 2 if the network was not used
                                because it was predicted not to pay (see nn_iter_ratio) */
    int32_t reserved;
} fg_result;

/* Defaults of SolverConfig::default() (crates/solver/src/lib.rs:116-120). */
FG_API void fg_cfg_default(fg_cfg *cfg);

/* Build the operator: uploads the mesh, computes the quadrature data
 * (PAMassOperator::new / PADiffusionOperator::new + the libCEED-style
 * qdata build of crates/assembly/src/reed/qfunction.rs:155-192 in 3-D).
 * kappa_q / rho_q: host or device arrays [E][qz][qy][qx] (E = nx*ny*nz, element index
 * (ez*ny + ey)*nx + ex) of per-quadrature-point coefficients, or NULL for the
 * constants.  nq1d must be order+1.  ess_tags: Dirichlet boundary tags used
 * when a call asks for the constrained operator. */
FG_API int fg_op_create(const fg_mesh *mesh, int order, int nq1d, int kind, double c_mass,
                        double c_diff, const double *kappa_q, double kappa_const,
                        const double *rho_q, double rho_const, int ess_tags, fg_op **out);
FG_API void fg_op_destroy(fg_op *op);

/* Build the operator on an unstructured Hex8 mesh with the caller's DOF
 * numbering: PAMassOperator::new / PADiffusionOperator::new(space, ...)
 * (crates/assembly/src/partial.rs:65-80, 138-149) for a space whose element
 * maps come from a DofManager (crates/space/src/dof_manager.rs:119-128), with
 * the essential DOFs of boundary_dofs (crates/space/src/constraints.rs:53-60)
 * as a list.  coords [n_nodes][3]; conn [n_elem][8] vertex ids in HexQ1 order
 * (crates/element/src/lagrange/hex.rs:27-36); elem_dofs [n_elem][(p+1)^3]:
 * order 1 in the HexQ1 vertex order, or NULL for DOF = node
 * (DofManager::build_p1); orders 2-3 in tensor order on the reference cube,
 * local DOF (c, b, a) at (c*(p+1) + b)*(p+1) + a, node (a, b, c) at
 * reference point (-1 + 2a/p, -1 + 2b/p, -1 + 2c/p) (the reference has no Q2/Q3
 * hex element; this is the equispaced tensor Lagrange element of this
 * library).  kappa_q / rho_q [n_elem][qz][qy][qx] at the tensor Gauss points
 * or NULL for the constants; ess_dofs [n_ess] (may repeat, order free).  All
 * arrays in host or device memory.  Geometry is trilinear from the 8
 * vertices (assembler.rs:96-143); a degenerate element gives FG_BOUNDS.
 * The native layout of the handle is the plain numbering padded with zeros
 * to a multiple of 4 values (fg_op_layout: {n_dofs, 1, 1, round_up(n_dofs, 4)}).  fg_op_apply,
 * fg_op_apply_native(_f32), fg_op_diagonal and fg_pcg (FG_PC_NONE, JACOBI,
 * CHEBYSHEV; FP64 and FG_FP32_IR) work as for a box; entry points that need
 * the box's lattice or tiles (affine format, tiles, batches, SDIRK-2, the
 * learned correction, the no-alloc apply) return FG_UNSUPPORTED.  The scatter
 * is chunked: elements in a Morton order form chunks of one CTA each, whose DOF
 * sums are formed in shared memory in a fixed order; DOFs shared between chunks
 * add their chunk partials in chunk order (no float atomics; the same sums
 * every run). */
FG_API int fg_op_create_hex(int order, int64_t n_nodes, const double *coords, int64_t n_elem,
                            const uint32_t *conn, const uint32_t *elem_dofs, int64_t n_dofs, int kind,
                            double c_mass, double c_diff, const double *kappa_q, double kappa_const,
                            const double *rho_q, double rho_const, const uint32_t *ess_dofs, int64_t n_ess,
                            fg_op **out);
/* Element chunks of an operator from fg_op_create_hex (0 for a box): the
 * elements in a Morton order of their centroids, one CTA per chunk, each
 * chunk's DOF sums formed in shared memory (no float atomics, no colour
 * passes). */
FG_API int64_t fg_op_chunks(const fg_op *op);

/* MatFreeOperator::n_dofs / LinearOperator::{nrows,ncols}. */
FG_API int64_t fg_op_ndofs(const fg_op *op);

/* dims = {NI, NJ, NK, NIp}: DOF grid and the native row pitch of device
 * vectors used by the *_native entry points (pads must hold zeros). */
FG_API int fg_op_layout(const fg_op *op, int64_t dims[4]);
FG_API int64_t fg_op_native_len(const fg_op *op);

/* Run on the caller's CUDA stream (cudaStream_t) instead of the handle's own. */
FG_API int fg_op_set_stream(fg_op *op, void *stream);

/* MatFreeOperator::apply (accumulate = 1: y += A x) and apply_zero
 * (accumulate = 0: y = A x); LinearOperator::apply is accumulate = 0.
 * constrained = 1 applies the Dirichlet elimination of the ess_tags DOFs
 * (rows and columns of essential DOFs replaced by the identity), the form the
 * solver uses.  x, y: plain lexicographic vectors of n_dofs doubles in host
 * (mem = FG_HOST) or device (FG_DEVICE) memory.  Synchronous.  Host vectors
 * go through a device staging buffer of n_dofs values that the first
 * host-memory call allocates; page-locked host memory runs the copies at full
 * PCIe rate.  With host vectors, accumulate = 0 and more than one layer of
 * work items in z, the call is pipelined over z ranges: the upload of the
 * next range's DOF planes, the apply of this range and the download of the
 * planes it finished run at the same time (the same sums as one launch).
 * Environment: FG_PIPELINED_APPLY=0 selects the serial form; FG_PIPE_RANGES
 * sets the number of z ranges (default 16, capped by the item layers). */
FG_API int fg_op_apply(fg_op *op, const double *x, double *y, int accumulate, int constrained,
                       int mem);

/* Same on device vectors in the native layout (fg_op_layout); asynchronous
 * on the handle's stream, no host synchronisation. */
FG_API int fg_op_apply_native(fg_op *op, const double *x, double *y, int accumulate,
                              int constrained);

/* Choose the quadrature-data format of the handle's applies and solves.
 * FG_QDATA_FULL (default): 6 symmetric components w|detJ| kappa J^-1 J^-T per
 * quadrature point (the general form of the reference's qdata,
 * crates/assembly/src/reed/qfunction.rs:155-192, in 3-D).  FG_QDATA_AFFINE:
 * valid only when J is constant over every element (parallelepipeds, e.g.
 * uniform boxes): 6 components of |detJ| J^-1 J^-T per element and one scalar
 * w kappa per quadrature point (plus w|detJ| rho for mass), about 5x fewer
 * bytes per apply.  Built from the full data on first use; returns
 * FG_UNSUPPORTED (format unchanged) when the mesh is not affine.  The Jacobi
 * diagonal and fg_op_apply_native_noalloc always use the full data. */
FG_API int fg_op_set_qdata_format(fg_op *op, int format);

/* FP32 form of the apply (the chosen precision form of the iterative
 * refinement): quadrature data rounded to FP32 once, FP32 vectors, FP32
 * arithmetic.  Same layouts and semantics as fg_op_apply / fg_op_apply_native
 * (MatFreeOperator::apply / apply_zero, crates/assembly/src/partial.rs:45-57). */
FG_API int fg_op_apply_f32(fg_op *op, const float *x, float *y, int accumulate, int constrained,
                           int mem);
FG_API int fg_op_apply_native_f32(fg_op *op, const float *x, float *y, int accumulate,
                                  int constrained);

/* fg_op_apply_native_noalloc: fg_op_apply_native without any device memory
 * management.  This entry point has no counterpart in the reference (fem-rs
 * has no GPU path); it exists for callers that cannot let a library allocate
 * device memory: programs whose memory pool or arena already owns the GPU's
 * memory (a cudaMalloc from here would fail or fragment their budget), and
 * loops that cannot afford the device-wide synchronisation that cudaMalloc
 * and cudaFree may imply.  The fix-up pass of the apply needs scratch for the
 * partial sums on tile faces; here that scratch is a fixed 32 MiB array
 * (4 Mi doubles) compiled into libfemgpu.so, which every GPU that loads the
 * library keeps until the process exits.  Operators whose face scratch
 * (about 0.22 * n_dofs doubles for Q2) exceeds it are rejected with
 * FG_INVALID_ARGUMENT.  The call allocates and frees nothing.  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress);
 * make that first call before any stream capture.  The address is tied to the
 * CUDA context: a call made in a different context of the device than the
 * last lookup (after cudaDeviceReset, or after the primary context was
 * released and created again) looks it up again.  All calls share the one
 * array: calls whose GPU work overlaps in time (other streams, other handles,
 * other threads) race on it and give wrong results; calls on one stream are
 * ordered and safe.  Nothing needs clearing between calls: every slot read is
 * written earlier in the same call.  Same vectors and semantics as
 * fg_op_apply_native. */
FG_API int fg_op_apply_native_noalloc(fg_op *op, const double *x, double *y, int accumulate,
                                      int constrained);

/* Diagonal of the (constrained) operator, 1 on essential DOFs (the Jacobi
 * diagonal CsrMatrix::diagonal gives after apply_dirichlet). */
FG_API int fg_op_diagonal(fg_op *op, double *d, int constrained, int mem);

/* Preconditioned CG on the constrained operator (solve_pcg_jacobi /
 * solve_cg_operator semantics): x holds the initial guess on entry and the
 * solution on exit.  Stopping rule of par_solve_pcg_jacobi, checked every
 * iteration on the device.  Returns FG_OK, FG_CONVERGENCE_FAILED or
 * FG_BREAKDOWN (res->status carries the same code). */
FG_API int fg_pcg(fg_op *op, const double *b, double *x, const fg_cfg *cfg, fg_result *res,
                  int mem);

/* Batched solves: n independent operators (any mix of orders and sizes)
 * solved together by the FP32 mixed-precision PCG of fg_pcg (cfg->precision
 * must be FG_FP32_IR; Jacobi or Chebyshev preconditioner).  Each phase of an
 * iteration is one launch over all instances (one per order/kind/format group
 * for the applies), converged instances are masked on the device, and chunks
 * of cfg->check_interval iterations are captured once in a CUDA graph and
 * replayed.  b[i], x[i]: plain vectors of operator i (x: guess in, solution
 * out); results[i] per instance.  Returns FG_CONVERGENCE_FAILED if any
 * instance did not converge.  No reference counterpart: fem-rs solves one
 * system per call (crates/solver/src/lib.rs:281-297). */
FG_API int fg_batch_pcg(fg_op *const *ops, int n, const double *const *b, double *const *x,
                        const fg_cfg *cfg, fg_result *results, int mem);

typedef struct {
    int32_t steps;
    int32_t max_stage_iterations;
    int64_t total_iterations;  /* PCG iterations over all stage solves */
    int32_t failed_solves;
    int32_t reserved;
    int64_t applies;
    double time_ms;            /* device time of the stepping loop */
} fg_sdirk_result;

/* SDIRK-2 heat stepping M u_t + K u = 0 with the constrained operators
 * (examples/mfem_ex10_heat_equation.rs:201-250; gamma = 1 - 1/sqrt(2),
 * crates/solver/src/ode.rs:441).  `stiff` is K (FG_DIFF); `stage` is
 * M + gamma*dt*K (FG_MASS_DIFF with c_mass = 1, c_diff = gamma*dt) on the same
 * mesh.  Each stage solves (M + gamma dt K) k = -K u_stage with fg_pcg's
 * solver and cfg, warm-started from the previous stage's k.  u: initial
 * condition in (zero on the Dirichlet DOFs), u(n_steps*dt) out. */
FG_API int fg_sdirk2(fg_op *stiff, fg_op *stage, double *u, double dt, int n_steps,
                     const fg_cfg *cfg, fg_sdirk_result *res, int mem);

/* ---- learned coarse correction ------------------------------------------
 * No reference counterpart (fem-rs has no learned components).  A small 3-D
 * U-net (3 levels, channels c0/c1/c2, default 16/32/48, ~250k parameters,
 * BF16 tensors with FP32 accumulation) maps a restricted residual and the
 * restricted log-coefficient to an error correction on the vertex grid
 * coarsened L = 1..4 times from an operator's DOF lattice (equispaced nodes
 * of any order form a uniform lattice; full-weighting R, trilinear P); with
 * FG_PC_CHEB_NN, fg_pcg runs flexible CG with
 * z = Chebyshev(r) + s 8^L P^L(UNet(R^L r / s, R^L log kappa)), s = rms(R^L r).
 * The convolutions run on the BF16 tensor cores through mma.sync.  Environment,
 * read by fg_unet_create: FG_UNET_TC=1 moves that network's forward and
 * input-gradient convolutions with channel counts that are multiples of 8 to
 * tcgen05 (accumulators in tensor memory); the mma.sync kernels measured
 * faster on the B200 at every volume from 9^3 to 2 x 65^3. */
typedef struct fg_unet fg_unet;
FG_API int fg_unet_create(const int channels[3], uint64_t seed, fg_unet **out);
FG_API void fg_unet_destroy(fg_unet *net);
FG_API int64_t fg_unet_num_params(const fg_unet *net);
/* Parameters / gradients as one FP32 array: per layer W[cout][27][cin] (tap =
 * (dz+1)*9 + (dy+1)*3 + (dx+1)), then b[cout]; layers in the order
 * l0a, l0b, l1a, l1b, l2a, l2b, l1c, l0c, out. */
FG_API int fg_unet_get_params(fg_unet *net, float *params);
FG_API int fg_unet_set_params(fg_unet *net, const float *params);
FG_API int fg_unet_get_grads(fg_unet *net, float *grads);
/* in: [B][Z][Y][X][2] FP32, out: [B][Z][Y][X] FP32 (channel 0); Z, Y, X = 1 mod 4, >= 5. */
FG_API int fg_unet_forward(fg_unet *net, const float *in, int B, int Z, int Y, int X, float *out, int mem);
/* mean squared error of output channel 0 against target [B][Z][Y][X] and its
 * gradients (no update) / one Adam step with learning rate lr. */
FG_API int fg_unet_loss_grad(fg_unet *net, const float *in, const float *target, int B, int Z, int Y,
                             int X, float *loss, int mem);
FG_API int fg_unet_train_step(fg_unet *net, const float *in, const float *target, int B, int Z, int Y,
                              int X, float lr, float *loss, int mem);
/* kappa at the DOFs (plain layout, host) for the log-coefficient channel and
 * the coarsening depth levels (1 to 4); the DOF lattice's cell counts
 * (p * elements per direction) must be multiples of 4 * 2^levels. */
FG_API int fg_op_set_nodal_kappa(fg_op *op, const double *kappa_nodal, int levels);
/* Attach (or with NULL detach) a network used by FG_PC_CHEB_NN. */
FG_API int fg_op_attach_unet(fg_op *op, fg_unet *net);
/* Training pairs from a plain Chebyshev-PCG solve (x0 = 0): at iterations
 * 0, every, 2*every, ... input [Zc][Yc][Xc][2] = (R r_k / s_k, R log kappa),
 * target [Zc][Yc][Xc] = (x* - x_k) at the coarse vertices / s_k, with
 * s_k = rms(R r_k); device FP32 buffers for max_pairs pairs. */
FG_API int fg_op_collect_pairs(fg_op *op, const double *b, const fg_cfg *cfg, int every, int max_pairs,
                               float *in, float *target, int *n_pairs);
/* Recurrence residuals of a plain Chebyshev-PCG solve (x0 = 0) at iterations
 * 0, every, 2*every, ...: device FP64, native layout, [max_res][native_len]. */
FG_API int fg_op_collect_residuals(fg_op *op, const double *b, const fg_cfg *cfg, int every, int max_res,
                                   double *res, int *n_res);
/* One Adam step on the energy loss of B residuals res (device, native layout,
 * [B][native_len], zero on essential DOFs): per sample c = s 8^L P^L UNet(...),
 * loss = (c.Ac/2 - c.r) / (s^2 64^L Nc), Nc = network voxels; its minimiser
 * over range(P^L) is the Galerkin coarse correction.  *loss = batch mean. */
FG_API int fg_unet_train_energy(fg_unet *net, fg_op *op, const double *res, int B, float lr, float *loss);

/* ---- tile shape and the batched autotuner ------------------------------------ */
/* An apply work item (one CTA's unit) is a box of 32 x WY x TZ elements; WY is
 * fixed per order, TZ (layers per item) is chosen at creation (8, halved until
 * there are >= 592 items) and can be changed: fg_op_set_tile re-lays out the
 * quadrature data on the device.  fg_op_tile returns {32, WY, TZ}.  No
 * reference counterpart (tuning of this library's kernels). */
FG_API int fg_op_set_tile(fg_op *op, int tz);
FG_API int fg_op_tile(const fg_op *op, int dims[3]);

#define FG_TUNE_CANDIDATES 5 /* TZ = 1, 2, 4, 8, 16 */
typedef struct {
    int32_t order, kind;
    int32_t format;      /* chosen quadrature-data format (FG_QDATA_FULL / FG_QDATA_AFFINE) */
    int32_t size_class;  /* 0: <= 16^3 elements, 1: <= 32^3, 2: larger */
    int32_t instances;   /* batch members in the class */
    int32_t tz;          /* chosen layers per item */
    double us[FG_TUNE_CANDIDATES];       /* batched FP32 apply time per TZ candidate in the chosen
                                            format, -1 = not tried */
    double us_other[FG_TUNE_CANDIDATES]; /* the same in the other format (-1: not tried, or the
                                            affine format refused by a member's geometry) */
} fg_tune_entry;
/* Autotuner for fg_batch_pcg: instances are grouped by (order, kind, size
 * class); for each group every candidate (quadrature-data format, TZ) -- the
 * affine format only when every member's elements have constant Jacobians;
 * TZ clamped per instance to the largest power of two <= nz -- is applied to
 * all members, the group's batched FP32 apply (one launch + fix-up) is timed
 * over `reps` launches with CUDA events, and the fastest pair is kept on the
 * operators (the FP64 reliable-update applies of the mixed solve use the same
 * format).  Results per group in out[0 .. min(*n_out, max_out)). */
FG_API int fg_batch_autotune(fg_op *const *ops, int n, int reps, fg_tune_entry *out, int max_out,
                             int *n_out);

/* ---- one-time work around the solve ---------------------------------------- */
/* Physical Gauss points (nq per direction, nq <= 8) of every element:
 * xyz[E][qz][qy][qx][3].  With nq = p+1 these are the points at which
 * kappa_q / rho_q / f_q tables are given. */
FG_API int fg_quadrature_points(const fg_mesh *mesh, int nq, double *xyz, int mem);
/* Linear form b_i = sum_e sum_q w_q |det J| f(x_q) phi_i(x_q) with the
 * (p+1)^3 Gauss rule: DomainSourceIntegrator + Assembler::assemble_linear
 * (crates/assembly/src/standard/source.rs:39-50, assembler.rs:251-333,
 * 434-454; hex_rule n = p+1 as in examples/mfem_ex1_poisson.rs:81,87).  f at
 * the Gauss points ([E][qz][qy][qx], host or device as mem) or NULL for the
 * constant f_const; the rows of the essential DOFs of ess_tags are set to
 * zero (apply_dirichlet with g = 0, crates/linalg/src/csr.rs:297-312). */
FG_API int fg_assemble_source(const fg_mesh *mesh, int order, const double *f_q, double f_const,
                              int ess_tags, double *b, int mem);
/* L2 norm of u_h - u with an nq-point Gauss rule per direction (nq <= 8):
 * u_h = the FE field of the DOF values u (plain layout), u at the Gauss points
 * ([E][nq^3]) or NULL for ||u_h||; the error norm of
 * examples/mfem_ex1_poisson.rs:119-162. */
FG_API int fg_l2_error(const fg_mesh *mesh, int order, int nq, const double *u, const double *u_q,
                       double *err, int mem);
/* LumpedMassOperator::assemble (crates/assembly/src/partial.rs:222-248): row-sum
 * lumped mass diag_i = sum_q w |det J| rho phi_i (sum_j phi_j), (p+1)^3 Gauss
 * rule, rho at the Gauss points or NULL for rho_const. */
FG_API int fg_lumped_mass(const fg_mesh *mesh, int order, const double *rho_q, double rho_const,
                          double *diag, int mem);
/* LumpedMassOperator apply (mode 1: y += d x), apply_zero (mode 0: y = d x) and
 * apply_inverse (mode 2: y = x / d, 0 where |d| <= 1e-14), partial.rs:251-273. */
FG_API int fg_lumped_apply(const double *diag, const double *x, double *y, int64_t n, int mode, int mem);

/* ---- tetrahedral PA operator -------------------------------------------------
 * PAMassOperator / PADiffusionOperator on Tet4 meshes with TetP1 / TetP2 / TetP3
 * (crates/assembly/src/partial.rs:85-130, 154-208 with ref_elem :277-288,
 * simplex_jac :290-299, xform_grads :301-309; bases
 * crates/element/src/lagrange/tet.rs; rule tet_rule(quad_order),
 * crates/element/src/quadrature.rs:259-376).  coords [n_nodes][3]; elem_dofs
 * [E][4 or 10] as DofManager numbers them (first 4 = vertex nodes,
 * crates/space/src/dof_manager.rs:137-180, 628-700); kappa_q / rho_q
 * [E][nq] at the rule's points (fg_tet_quadrature_points) or NULL for the
 * constants; ess: essential-DOF mask [n_dofs] (boundary_dofs) or NULL.  TetP3
 * element maps: [E][20] as build_p3_tet (dof_manager.rs:484-600).  All
 * arrays in host or device memory.  The scatter is the transpose of the
 * element map summed in a fixed order (no float atomics). */
typedef struct fg_tet fg_tet;
FG_API int fg_tet_create(int order, int64_t n_nodes, const double *coords, int64_t n_elem,
                         const int32_t *elem_dofs, int64_t n_dofs, int kind, double c_mass, double c_diff,
                         const double *kappa_q, double kappa_const, const double *rho_q, double rho_const,
                         int quad_order, const uint8_t *ess, fg_tet **out);
FG_API void fg_tet_destroy(fg_tet *op);
FG_API int64_t fg_tet_ndofs(const fg_tet *op);
/* quadrature points per element of the operator's rule */
FG_API int fg_tet_nq(const fg_tet *op);
/* physical quadrature points xyz[E][nq][3] = x_0 + J xi_q */
FG_API int fg_tet_quadrature_points(fg_tet *op, double *xyz, int mem);
/* MatFreeOperator::apply (accumulate = 1) / apply_zero (0); constrained = 1:
 * identity rows and columns on the essential DOFs. */
FG_API int fg_tet_apply(fg_tet *op, const double *x, double *y, int accumulate, int constrained, int mem);
/* Jacobi diagonal (1 on essential DOFs when constrained). */
FG_API int fg_tet_diagonal(fg_tet *op, double *d, int constrained, int mem);
/* fg_tet_apply on device vectors, asynchronous on the handle's stream (no
 * host synchronisation). */
FG_API int fg_tet_apply_native(fg_tet *op, const double *x, double *y, int accumulate, int constrained);
/* Run on the caller's CUDA stream (cudaStream_t) instead of the handle's own. */
FG_API int fg_tet_set_stream(fg_tet *op, void *stream);
/* Synchronise the handle's stream. */
FG_API int fg_tet_check(fg_tet *op);

/* Limit of each device-side wait of this handle's apply kernels for a copy
 * into shared memory (default 1 s; seconds <= 0 restores it, at most 60 s).
 * A wait that runs out sets the handle's device error word, the kernel stops
 * issuing copies, waits (1 s at most each) for the copies it has in flight and
 * returns; fg_op_check then reports FG_DEVICE_TIMEOUT and clears the word.
 * The results of an apply that timed out are not defined.  No reference
 * counterpart (the reference has no device code); a watchdog for the hosts of
 * this library. */
FG_API int fg_op_set_wait_limit(fg_op *op, double seconds);

/* Steps of a PCG whose dot products are completed by the caller, on device
 * vectors of the handle's native layout (fg_op_native_len values), on the
 * handle's stream, scalars in device memory: the sharded solve of
 * par_solve_pcg_jacobi (crates/parallel/src/par_solver.rs:262-342), where each
 * rank reduces over the DOFs it owns and an allreduce adds the ranks' sums
 * (ParVector::global_dot, crates/parallel/src/par_vector.rs:182-194).  The
 * owned DOFs are the prefix [0, n_own) of the local vector, n_own a multiple
 * of 4.  Reductions are summed in a fixed order (the same bits every run).
 *   fg_vec_dots:       out[j] = a_j . b_j over the owned prefix, j < npairs <= 3
 *   fg_vec_pcg_update: alpha = rz_pap[0] / rz_pap[1]; x += alpha p,
 *                      r -= alpha ap, z = dinv r (whole vector);
 *                      rr_rz = (r . r, r . z) over the owned prefix
 *   fg_vec_pupdate:    p = z + (*num / *den) p */
FG_API int fg_vec_dots(fg_op *op, int64_t n_own, int npairs, const double *const *a, const double *const *b,
                       double *out);
FG_API int fg_vec_pcg_update(fg_op *op, int64_t n_own, double *x, double *r, const double *p, const double *ap,
                             const double *dinv, double *z, const double *rz_pap, double *rr_rz);
FG_API int fg_vec_pupdate(fg_op *op, const double *z, double *p, const double *num, const double *den);

/* Synchronise the handle's stream and report device-side errors
 * (FG_DEVICE_TIMEOUT, FG_BOUNDS). */
FG_API int fg_op_check(fg_op *op);

/* Message of the last failing call on this thread; returns its status. */
FG_API int fg_last_error(char *buf, size_t n);

#ifdef __cplusplus
}
#endif
#endif
