"""GPU parity of the sm_100a PA operator, diagonal and PCG against the CPU
oracle (the restated reference algorithm), through the C ABI.

Tolerance: the north-star bar, 1e-12 relative error (2-norm) of the FP64 apply
against the oracle on identical meshes and inputs; PCG iteration counts within
+-1 of the oracle's.
"""
import numpy as np
import pytest

from conftest import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import femgpu  # noqa: E402
from femgpu.fields import lognormal_kappa_q  # noqa: E402

RTOL = 1e-12


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def perturbed_vertices(nx, ny, nz, amp=0.15, seed=0):
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    v = np.stack([i / nx, j / ny, k / nz], axis=-1).astype(np.float64)
    h = np.array([1 / nx, 1 / ny, 1 / nz])
    interior = (i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)
    v[interior] += amp * h * rng.uniform(-1, 1, size=(interior.sum(), 3))
    return v.reshape(-1, 3)


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def make_pair(shape, p, kind, seed=0, perturb=True, kappa_field=True, ess=femgpu.TAG_ALL,
              c_m=1.0, c_k=1.0):
    nx, ny, nz = shape
    vc = perturbed_vertices(nx, ny, nz, seed=seed) if perturb else None
    rng = np.random.default_rng(100 + seed)
    E, q3 = nx * ny * nz, (p + 1) ** 3
    kq = np.exp(rng.normal(size=E * q3)) if kappa_field else None
    rq = np.exp(0.3 * rng.normal(size=E * q3)) if kappa_field else None
    mesh = O.Mesh(nx, ny, nz, p, vcoord=vc)
    coef = O.Coef(kind, c_m=c_m, c_k=c_k, kappa_q=kq, kappa=1.0, rho_q=rq, rho=1.0)
    gm = dict(nx=nx, ny=ny, nz=nz, vcoord=vc)
    op = femgpu.PAOperator(gm, p, kind, kappa=kq if kq is not None else 1.0,
                           rho=rq if rq is not None else 1.0, c_mass=c_m, c_diff=c_k, ess_tags=ess)
    return mesh, coef, op


# shapes chosen to cover single/multiple tiles in x (32 elements), y and z
SHAPES = [(1, 1, 1), (3, 2, 2), (7, 5, 9), (33, 6, 5), (40, 9, 17)]


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("kind", [femgpu.MASS, femgpu.DIFF, femgpu.MASS_DIFF])
@pytest.mark.parametrize("shape", SHAPES)
def test_apply_matches_oracle(p, kind, shape):
    need_gpu()
    if p == 3 and shape[0] * shape[1] * shape[2] > 2000:
        shape = (33, 3, 3)
    mesh, coef, op = make_pair(shape, p, kind, seed=sum(shape) + p, c_m=1.7, c_k=0.9)
    x = np.random.default_rng(7).normal(size=mesh.ndofs)
    y_ref = O.pa_apply(mesh, coef, x)
    y = op.matvec(x)
    assert relerr(y, y_ref) <= RTOL, relerr(y, y_ref)
    # accumulate form: y += A x
    y2 = y.copy()
    op.apply(x, y2)
    assert relerr(y2, 2 * y_ref) <= RTOL


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("ess", [femgpu.TAG_ALL, 1 | 16, 32 | 8])
def test_constrained_apply_and_diagonal(p, ess):
    need_gpu()
    shape = (35, 6, 10) if p < 3 else (33, 3, 4)
    mesh, coef, op = make_pair(shape, p, femgpu.DIFF, seed=p, ess=ess)
    mask = O.ess_mask(mesh, ess)
    x = np.random.default_rng(3).normal(size=mesh.ndofs)
    y_ref = O.apply_constrained(mesh, coef, mask, x)
    y = op.matvec(x, constrained=True)
    assert relerr(y, y_ref) <= RTOL
    d_ref = O.diagonal(mesh, coef, mask)
    d = op.diagonal(constrained=True)
    assert relerr(d, d_ref) <= RTOL
    d0 = op.diagonal(constrained=False)
    assert relerr(d0, O.diagonal(mesh, coef, None)) <= RTOL


def test_apply_is_deterministic_and_device_pointers_work():
    need_gpu()
    mesh, coef, op = make_pair((40, 9, 17), 2, femgpu.DIFF, seed=5)
    x = np.random.default_rng(11).normal(size=mesh.ndofs)
    a, b = op.matvec(x), op.matvec(x)
    assert np.array_equal(a, b)
    xt = torch.from_numpy(x).cuda()
    yt = torch.zeros_like(xt)
    op.apply_zero(xt, yt)
    assert np.array_equal(yt.cpu().numpy(), a)


@pytest.mark.parametrize("p,shape", [(1, (70, 9, 11)), (2, (40, 9, 17)), (3, (33, 5, 6))])
def test_fused_fixup_option_is_bit_identical(p, shape, monkeypatch):
    """FG_FUSED_FIXUP=1 (the fix-up done by the last contributing item inside
    the apply kernel, a run-time option) gives the same bits as the separate
    fix-up kernel, FP64 and FP32, raw and constrained, on multi-item grids."""
    need_gpu()
    mesh, coef, op = make_pair(shape, p, femgpu.MASS_DIFF, seed=9)
    monkeypatch.setenv("FG_FUSED_FIXUP", "1")
    _, _, fused = make_pair(shape, p, femgpu.MASS_DIFF, seed=9)
    monkeypatch.delenv("FG_FUSED_FIXUP")
    x = np.random.default_rng(3).normal(size=mesh.ndofs)
    for constrained in (False, True):
        for _ in range(2):  # the arrival counters reset themselves between launches
            assert np.array_equal(fused.matvec(x, constrained=constrained), op.matvec(x, constrained=constrained))
    xn = torch.from_numpy(op.to_native(x)).float().cuda()
    ya, yb = torch.zeros_like(xn), torch.zeros_like(xn)
    torch.cuda.synchronize()
    op.apply_native_f32(xn.data_ptr(), ya.data_ptr())
    fused.apply_native_f32(xn.data_ptr(), yb.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(ya, yb)
    op.close()
    fused.close()


def test_native_layout_apply_matches_plain():
    need_gpu()
    mesh, coef, op = make_pair((33, 5, 6), 2, femgpu.MASS_DIFF, seed=2)
    x = np.random.default_rng(4).normal(size=mesh.ndofs)
    xn = torch.from_numpy(op.to_native(x)).cuda()
    yn = torch.zeros_like(xn)
    op.apply_native(xn.data_ptr(), yn.data_ptr(), accumulate=False, constrained=False)
    torch.cuda.synchronize()
    ynh = yn.cpu().numpy()
    assert np.array_equal(op.from_native(ynh), op.matvec(x))
    pads = ynh.reshape(op.NK, op.NJ, op.NIp)[:, :, op.NI:]
    assert not pads.any()


def test_reference_known_answers_on_gpu():
    """partial.rs:380-392 (K 1 = 0), standard/mass.rs:67-82 (1'M1 = |Omega|)."""
    need_gpu()
    for p in (1, 2, 3):
        vc = perturbed_vertices(4, 3, 3, seed=p)
        opk = femgpu.PADiffusionOperator(dict(nx=4, ny=3, nz=3, vcoord=vc), p)
        one = np.ones(opk.n_dofs())
        assert np.abs(opk.matvec(one)).max() < 1e-12
        opm = femgpu.PAMassOperator(dict(nx=4, ny=3, nz=3, vcoord=vc), p)
        assert abs(one @ opm.matvec(one) - 1.0) < 1e-10


def test_pcg_jacobi_matches_oracle_iterations_c0():
    """Poisson on 24^3 Q1, kappa = 1, PCG-Jacobi, rtol 1e-10 (mfem_ex1 template)."""
    need_gpu()
    n = 24
    mesh = O.Mesh(n, n, n, 1)
    mask = O.ess_mask(mesh)
    b = O.source(mesh, mask)
    coef = O.Coef(O.DIFF)
    x_ref, info = O.pcg(mesh, coef, mask, b, precond=1, rtol=1e-10, max_iter=5000)
    op = femgpu.PADiffusionOperator((n, n, n), 1)
    x = np.zeros(mesh.ndofs)
    res = femgpu.solve_pcg_jacobi(op, b, x, femgpu.SolverConfig(rtol=1e-10, max_iter=5000))
    assert res.converged and info["converged"]
    assert abs(res.iterations - info["iterations"]) <= 1, (res.iterations, info["iterations"])
    assert res.true_residual < 1e-10 * 1.01
    assert relerr(x, x_ref) < 1e-8
    assert O.l2_error_sin(mesh, x) < 2.2e-2


@pytest.mark.parametrize("p", [1, 2, 3])
def test_pcg_chebyshev_matches_oracle(p):
    need_gpu()
    n = {1: 12, 2: 8, 3: 6}[p]
    rng = np.random.default_rng(p)
    kq = np.exp(rng.normal(size=n ** 3 * (p + 1) ** 3))
    mesh = O.Mesh(n, n, n, p)
    mask = O.ess_mask(mesh)
    coef = O.Coef(O.DIFF, kappa_q=kq)
    b = O.source(mesh, mask)
    lmax_ref = O.lambda_max(mesh, coef, mask, iters=20)
    x_ref, info = O.pcg(mesh, coef, mask, b, precond=2, cheb_degree=4, lmin=1.1 * lmax_ref / 30,
                        lmax=1.1 * lmax_ref, rtol=1e-8)
    op = femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
    x = np.zeros(mesh.ndofs)
    res = femgpu.solve_pcg_chebyshev(op, b, x, femgpu.SolverConfig(rtol=1e-8, cheb_degree=4))
    assert abs(res.lmax - 1.1 * lmax_ref) <= 1e-10 * lmax_ref
    assert res.converged and abs(res.iterations - info["iterations"]) <= 1
    assert res.true_residual <= 1e-8 * 1.05
    assert relerr(x, x_ref) < 1e-6


def test_cg_operator_errors():
    need_gpu()
    op = femgpu.PADiffusionOperator((4, 4, 4), 1)
    n = op.n_dofs()
    with pytest.raises(femgpu.DimensionMismatch):
        femgpu.solve_cg_operator(n, n + 1, op, np.ones(n), np.zeros(n))
    b = np.random.default_rng(0).normal(size=n)
    with pytest.raises(femgpu.ConvergenceFailed):
        femgpu.solve_cg_operator(n, n, op, b, np.zeros(n), femgpu.SolverConfig(rtol=1e-14, max_iter=3))
    x = np.zeros(n)
    res = femgpu.solve_cg_operator(n, n, op, b, x, femgpu.SolverConfig(rtol=1e-10, max_iter=500))
    assert res.converged and res.true_residual < 1e-9


def test_zero_rhs_returns_immediately():
    need_gpu()
    op = femgpu.PADiffusionOperator((5, 5, 5), 2)
    n = op.n_dofs()
    x = np.zeros(n)
    res = femgpu.solve_pcg_jacobi(op, np.zeros(n), x)
    assert res.converged and res.iterations == 0 and not x.any()


@pytest.mark.parametrize("rtol,atol", [(1e-9, 0.0), (1e-12, 1e-4)])
def test_cg_operator_stopping_rule_matches_oracle(rtol, atol):
    """FG_PC_NONE is solve_cg_operator (crates/solver/src/lib.rs:229-278):
    ||r|| <= max(atol, rtol*max(||b||, 1e-32)), absolute final residual,
    exit before the first iteration when the start already meets it."""
    need_gpu()
    n, p = 6, 2
    kq = lognormal_kappa_q(n, n, n, p, seed=8)
    mesh = O.Mesh(n, n, n, p)
    mask = O.ess_mask(mesh)
    b = O.source(mesh, mask)
    _, info = O.pcg(mesh, O.Coef(O.DIFF, kappa_q=kq), mask, b, precond=0, rtol=rtol, atol=atol, max_iter=5000)
    op = femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
    N = op.n_dofs()
    x = np.zeros(N)
    res = femgpu.solve_cg_operator(N, N, op, b, x, femgpu.SolverConfig(rtol=rtol, atol=atol, max_iter=5000))
    assert res.converged and abs(res.iterations - info["iterations"]) <= 1
    tol = max(atol, rtol * np.linalg.norm(b))
    assert 0.05 * tol < res.final_residual <= tol
    # restart from the solution with a tolerance it already meets
    res0 = femgpu.solve_cg_operator(N, N, op, b, x.copy(),
                                    femgpu.SolverConfig(rtol=0.0, atol=2.0 * res.final_residual))
    assert res0.converged and res0.iterations == 0


@pytest.mark.parametrize("p,shape", [(1, (70, 9, 40)), (2, (40, 9, 37)), (3, (33, 5, 26)), (2, (128, 16, 64))])
def test_pipelined_host_apply_is_bit_identical(p, shape, monkeypatch):
    """fg_op_apply on host vectors runs in z ranges of item layers (upload of the
    next range, apply and fix-up of this one, download of the finished planes
    overlapped); the sums are those of the one-launch apply, bit for bit."""
    need_gpu()
    mesh, coef, op = make_pair(shape, p, femgpu.MASS_DIFF, seed=3, c_m=0.4, c_k=1.2)
    monkeypatch.setenv("FG_PIPELINED_APPLY", "0")
    _, _, ref = make_pair(shape, p, femgpu.MASS_DIFF, seed=3, c_m=0.4, c_k=1.2)
    monkeypatch.delenv("FG_PIPELINED_APPLY")
    assert op.tile[2] < shape[2]  # more than one item layer: the pipelined path runs
    x = np.random.default_rng(8).normal(size=mesh.ndofs)
    for constrained in (False, True):
        for _ in range(2):
            assert np.array_equal(op.matvec(x, constrained=constrained), ref.matvec(x, constrained=constrained))
    assert relerr(op.matvec(x, constrained=True), O.apply_constrained(mesh, coef, O.ess_mask(mesh), x)) <= RTOL
    op.close()
    ref.close()
