"""Error paths of the C ABI on the GPU, each made on the host side (bad input
data, never a device fault).

* A NaN in the right-hand side or the initial guess: the reference's CG loops
  never meet their stopping test on NaN residuals and end with
  ConvergenceFailed (crates/solver/src/lib.rs:243-277,
  crates/parallel/src/par_solver.rs:296-341); the library returns
  FG_CONVERGENCE_FAILED or FG_BREAKDOWN, never FG_OK, and the handle stays
  usable for the next solve.
* p^T A p below the breakdown threshold: solve_cg_operator returns
  SolverError::Linger("CG operator breakdown ...") (lib.rs:243-249); here
  FG_BREAKDOWN, raised as femgpu.Breakdown.
* A collapsed hexahedron (det J = 0 at its quadrature points): the
  reference's assembler panics on the singular Jacobian
  (crates/assembly/src/assembler.rs:223-225); fg_op_create returns FG_BOUNDS
  and no handle.
"""
import numpy as np
import pytest

from conftest import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import femgpu  # noqa: E402


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _problem(n=8, p=2):
    op = femgpu.PADiffusionOperator((n, n, n), p)
    mesh = O.Mesh(n, n, n, p)
    mask = O.ess_mask(mesh)
    b = O.source(mesh, mask)
    return op, b


@pytest.mark.parametrize("where", ["rhs", "guess"])
@pytest.mark.parametrize("precond", [femgpu.PC_NONE, femgpu.PC_JACOBI, femgpu.PC_CHEBYSHEV])
@pytest.mark.parametrize("precision", [femgpu.FP64, femgpu.FP32_IR])
def test_nan_input_fails_and_handle_stays_usable(where, precond, precision):
    need_gpu()
    if precond == femgpu.PC_NONE and precision == femgpu.FP32_IR:
        pytest.skip("the operator CG runs in FP64 only")
    op, b = _problem()
    N = op.n_dofs()
    bad_b, x0 = b.copy(), np.zeros(N)
    idx = N // 2 + 3  # an interior DOF
    if where == "rhs":
        bad_b[idx] = np.nan
    else:
        x0[idx] = np.nan
    cfg = femgpu.SolverConfig(rtol=1e-8, max_iter=40, precision=precision)
    try:
        res = op.pcg(bad_b, x0, cfg, precond)
        assert not res.converged
        assert res.status == femgpu.FG_CONVERGENCE_FAILED, res.status
    except femgpu.Breakdown:
        pass
    # the same handle solves a clean problem afterwards
    x = np.zeros(N)
    ok = op.pcg(b, x, femgpu.SolverConfig(rtol=1e-8, max_iter=2000, precision=precision),
                femgpu.PC_JACOBI if precond == femgpu.PC_NONE else precond)
    assert ok.converged and ok.true_residual <= 1.05e-8
    op.check()
    op.close()


def test_operator_cg_breakdown():
    """p^T A p ~ 1e-46 < 1e-32 from the first iteration: Breakdown, as
    solve_cg_operator's Linger error."""
    need_gpu()
    n, p = 6, 1
    op = femgpu.PAOperator((n, n, n), p, femgpu.MASS, c_mass=1e-40)
    mesh = O.Mesh(n, n, n, p)
    mask = O.ess_mask(mesh).astype(bool)
    b = np.random.default_rng(0).standard_normal(mesh.ndofs)
    b[mask] = 0.0
    x = np.zeros(mesh.ndofs)
    with pytest.raises(femgpu.Breakdown):
        femgpu.solve_cg_operator(mesh.ndofs, mesh.ndofs, op, b, x, femgpu.SolverConfig(rtol=1e-8, max_iter=50))
    op.close()


@pytest.mark.parametrize("order", [1, 2, 3])
def test_collapsed_hex_is_rejected(order):
    """The vertex plane k = 1 moved onto k = 0: the first element layer has
    zero thickness, det J = 0 exactly at every quadrature point."""
    need_gpu()
    nx, ny, nz = 3, 2, 2
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    vc = np.stack([i / nx, j / ny, k / nz], axis=-1).astype(np.float64)
    vc[1, :, :, 2] = 0.0
    with pytest.raises(femgpu.SolverError) as exc:
        femgpu.PADiffusionOperator(dict(nx=nx, ny=ny, nz=nz, vcoord=vc.reshape(-1, 3)), order)
    assert exc.value.status == femgpu.FG_BOUNDS
    assert "degenerate" in str(exc.value)
    # a valid mesh still builds afterwards
    op = femgpu.PADiffusionOperator((nx, ny, nz), order)
    assert np.abs(op.matvec(np.ones(op.n_dofs()))).max() < 1e-12
    op.close()


def test_device_wait_limit_runs_out_and_handle_recovers():
    """A 1 ns limit on the apply kernel's waits for its bulk copies makes them
    run out (a copy from HBM takes far longer): the kernel stops issuing,
    waits out the copies it has in flight with the normal limit, returns, and
    fg_op_check reports FG_DEVICE_TIMEOUT.  With the default limit restored
    the same handle applies correctly again."""
    need_gpu()
    n, p = 64, 2
    op = femgpu.PADiffusionOperator((n, n, n), p)
    x = np.random.default_rng(4).standard_normal(op.n_dofs())
    xt = torch.from_numpy(op.to_native(x)).cuda()
    yt = torch.zeros_like(xt)
    torch.cuda.synchronize()
    op.set_wait_limit(1e-9)
    status = femgpu.FG_OK
    for _ in range(10):
        op.apply_native(xt.data_ptr(), yt.data_ptr(), accumulate=False, constrained=True)
        try:
            op.check()
        except femgpu.SolverError as exc:
            status = exc.status
            break
    assert status == femgpu.FG_DEVICE_TIMEOUT, status
    op.set_wait_limit(0)
    mesh = O.Mesh(n, n, n, p)
    y_ref = O.apply_constrained(mesh, O.Coef(O.DIFF), O.ess_mask(mesh), x)
    y = op.matvec(x, constrained=True)
    op.check()
    assert np.linalg.norm(y - y_ref) <= 1e-12 * np.linalg.norm(y_ref)
    op.close()
