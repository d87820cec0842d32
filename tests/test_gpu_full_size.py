"""GPU parity at the benchmark sizes, through the C ABI, against the oracle on
the whole mesh.

The operators are exactly those the benchmark times: the unit-cube 128^3 Q2
mesh (257^3 = 16,974,593 DOFs, 3^3 Gauss points) and the 64^3 Q3 mesh
(193^3 = 7,189,057 DOFs, 4^3 Gauss points), kappa = exp(g) with g the
squared-exponential Gaussian field (sigma^2 = 1, correlation length 0.1,
seed 0) at the Gauss points, item tiling chosen by the library for these sizes
(the quadrature-data layout of the timed runs).  The oracle restates the
reference's element loop (crates/assembly/src/partial.rs:154-208 with the Hex8
Jacobian of crates/assembly/src/assembler.rs:96-143) and applies the full
mesh in about a second on the host cores.

Tolerances: FP64 applies and the Jacobi diagonal 1e-12 relative (2-norm), the
north-star bar; FP32 applies 2e-5 relative (FP32 rounding of the data and the
arithmetic, as in the smaller FP32 tests).

Also here: PCG iteration counts within +-1 of the oracle's on problems that
take tens to hundreds of iterations (crates/parallel/src/par_solver.rs:262-342
for Jacobi, Chebyshev(4) on D^-1 A for the scale-up configuration's solver).
"""
import numpy as np
import pytest

from conftest import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import femgpu  # noqa: E402
from femgpu.fields import lognormal_kappa_q, sin_nodal  # noqa: E402

RTOL64 = 1e-12
RTOL32 = 2e-5


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def relerr(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _f32_apply(op, x):
    """FP32 constrained apply of the handle's current format on a device vector."""
    xn = torch.from_numpy(op.to_native(x)).float().cuda()
    yn = torch.zeros_like(xn)
    torch.cuda.synchronize()
    op.apply_native_f32(xn.data_ptr(), yn.data_ptr(), accumulate=False, constrained=True)
    torch.cuda.synchronize()
    op.check()
    return op.from_native(yn.double().cpu().numpy())


@pytest.mark.parametrize("n,p", [(128, 2), (64, 3)], ids=["q2_128", "q3_64"])
def test_benchmark_operator_matches_oracle(n, p):
    need_gpu()
    kq = lognormal_kappa_q(n, n, n, p, sigma2=1.0, ell=0.1, seed=0)
    mesh = O.Mesh(n, n, n, p)
    coef = O.Coef(O.DIFF, kappa_q=kq)
    mask = O.ess_mask(mesh)
    op = femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
    assert op.n_dofs() == mesh.ndofs == (n * p + 1) ** 3
    x = np.random.default_rng(1000).standard_normal(mesh.ndofs)

    # raw operator (MatFreeOperator::apply_zero) and the constrained one the
    # solver and the benchmark use, FP64 full-format quadrature data
    y_ref = O.pa_apply(mesh, coef, x)
    e_raw = relerr(op.matvec(x), y_ref)
    assert e_raw <= RTOL64, e_raw
    yc_ref = O.apply_constrained(mesh, coef, mask, x)
    e_con = relerr(op.matvec(x, constrained=True), yc_ref)
    assert e_con <= RTOL64, e_con
    # the benchmark's call: native-layout device vectors on the caller's stream
    xn = torch.from_numpy(op.to_native(x)).cuda()
    yn = torch.zeros_like(xn)
    stream = torch.cuda.current_stream()
    op.set_stream(stream.cuda_stream)
    torch.cuda.synchronize()
    op.apply_native(xn.data_ptr(), yn.data_ptr(), accumulate=False, constrained=True)
    torch.cuda.synchronize()
    op.check()
    e_nat = relerr(op.from_native(yn.cpu().numpy()), yc_ref)
    assert e_nat <= RTOL64, e_nat
    del xn, yn

    # Jacobi diagonal of the constrained operator
    e_d = relerr(op.diagonal(constrained=True), O.diagonal(mesh, coef, mask))
    assert e_d <= RTOL64, e_d

    # FP32 apply on the full format
    e32 = relerr(_f32_apply(op, x), yc_ref)
    assert e32 <= RTOL32, e32

    # affine-compressed format (valid: the uniform mesh has constant J per
    # element), FP64 and FP32, against the same oracle result
    op.set_qdata_format(femgpu.QDATA_AFFINE)
    e_aff = relerr(op.matvec(x, constrained=True), yc_ref)
    assert e_aff <= RTOL64, e_aff
    e_aff32 = relerr(_f32_apply(op, x), yc_ref)
    assert e_aff32 <= RTOL32, e_aff32
    op.close()


def _dirichlet_zero(b, mask):
    b = b.copy()
    b[mask.astype(bool)] = 0.0
    return b


@pytest.mark.parametrize("case", ["random_rhs", "perturbed_lognormal"])
def test_pcg_jacobi_iterations_c0_mesh(case):
    """24^3 Q1 (the mfem_ex1 mesh), PCG-Jacobi to rtol 1e-10.  With the
    manufactured sine load both sides converge in one iteration (the load is an
    eigenvector of D^-1 A on the uniform grid), which checks nothing; these
    right-hand sides and coefficients take hundreds of iterations."""
    need_gpu()
    n, p = 24, 1
    rng = np.random.default_rng(24)
    if case == "random_rhs":
        vc, kq = None, None
    else:
        k, j, i = np.meshgrid(np.arange(n + 1), np.arange(n + 1), np.arange(n + 1), indexing="ij")
        vc = np.stack([i / n, j / n, k / n], axis=-1).astype(np.float64)
        inner = (i > 0) & (i < n) & (j > 0) & (j < n) & (k > 0) & (k < n)
        vc[inner] += 0.2 / n * rng.uniform(-1, 1, size=(inner.sum(), 3))
        vc = vc.reshape(-1, 3)
        kq = lognormal_kappa_q(n, n, n, p, seed=5)
    mesh = O.Mesh(n, n, n, p, vcoord=vc)
    mask = O.ess_mask(mesh)
    coef = O.Coef(O.DIFF, kappa_q=kq)
    b = _dirichlet_zero(rng.standard_normal(mesh.ndofs), mask)
    x_ref, info = O.pcg(mesh, coef, mask, b, precond=1, rtol=1e-10, max_iter=5000)
    assert info["converged"] and info["iterations"] > 30, info
    op = femgpu.PADiffusionOperator(dict(nx=n, ny=n, nz=n, vcoord=vc), p,
                                    kappa=1.0 if kq is None else kq)
    x = np.zeros(mesh.ndofs)
    res = femgpu.solve_pcg_jacobi(op, b, x, femgpu.SolverConfig(rtol=1e-10, max_iter=5000))
    assert res.converged
    assert abs(res.iterations - info["iterations"]) <= 1, (res.iterations, info["iterations"])
    assert res.true_residual < 1.05e-10
    assert relerr(x, x_ref) < 1e-7
    op.close()


@pytest.mark.parametrize("n,p", [(32, 2), (16, 3)], ids=["q2_32", "q3_16"])
def test_pcg_chebyshev_iterations_lognormal(n, p):
    """The scale-up configuration's solver (Chebyshev(4) on D^-1 A, lambda_max
    = 1.1 x 20 power iterations, lambda_min = lambda_max / 30, FP64 residual
    1e-8) with its lognormal kappa and load, on meshes the oracle solves in
    seconds: iterations within +-1."""
    need_gpu()
    kq = lognormal_kappa_q(n, n, n, p, sigma2=1.0, ell=0.1, seed=3)
    mesh = O.Mesh(n, n, n, p)
    mask = O.ess_mask(mesh)
    coef = O.Coef(O.DIFF, kappa_q=kq)
    mass = femgpu.PAMassOperator((n, n, n), p)
    b = _dirichlet_zero(mass.matvec(sin_nodal(n, n, n, p)), mask)
    mass.close()
    lmax_ref = O.lambda_max(mesh, coef, mask, iters=20)
    x_ref, info = O.pcg(mesh, coef, mask, b, precond=2, cheb_degree=4, lmin=1.1 * lmax_ref / 30,
                        lmax=1.1 * lmax_ref, rtol=1e-8, max_iter=5000)
    assert info["converged"] and info["iterations"] > 20, info
    op = femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
    x = np.zeros(mesh.ndofs)
    res = femgpu.solve_pcg_chebyshev(op, b, x, femgpu.SolverConfig(rtol=1e-8, cheb_degree=4, max_iter=5000))
    assert abs(res.lmax - 1.1 * lmax_ref) <= 1e-10 * lmax_ref
    assert res.converged
    assert abs(res.iterations - info["iterations"]) <= 1, (res.iterations, info["iterations"])
    assert res.true_residual <= 1.05e-8
    assert relerr(x, x_ref) < 1e-6
    op.close()
