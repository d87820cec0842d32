"""Batched uneven solves (fg_batch_pcg): mixed orders and sizes in one launch
per phase, per-instance convergence masks, CUDA-graph replay.

Each instance must meet the FP64 true-residual target (rtol 1e-8), agree with
the oracle's FP64 solution to 1e-7 relative, and take
the same number of iterations as solving that instance alone (+-2: the batched
reductions use a different, still fixed, partial-sum grid).
"""
import numpy as np
import pytest

from conftest import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import femgpu  # noqa: E402
from femgpu.fields import lognormal_kappa_q  # noqa: E402


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def make_instances(specs, seed=0):
    rng = np.random.default_rng(seed)
    inst = []
    for i, (n, p) in enumerate(specs):
        kq = lognormal_kappa_q(n, n, n, p, sigma2=float(rng.uniform(0.25, 2.0)),
                               ell=float(rng.uniform(0.05, 0.3)), seed=seed * 1000 + i)
        mesh = O.Mesh(n, n, n, p)
        mask = O.ess_mask(mesh)
        xi = rng.standard_normal(mesh.ndofs)
        b = O.pa_apply(mesh, O.Coef(O.MASS), xi)  # i.i.d. nodal values projected onto M
        b[mask == 1] = 0.0
        op = femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
        inst.append((mesh, mask, kq, b, op))
    return inst


SPECS = [(3, 1), (7, 2), (5, 3), (12, 1), (4, 2), (9, 2), (2, 3), (33, 1), (6, 1), (3, 2)]


@pytest.mark.parametrize("precond", [femgpu.PC_CHEBYSHEV, femgpu.PC_JACOBI])
def test_batched_solves_match_oracle_and_single_solves(precond):
    need_gpu()
    inst = make_instances(SPECS, seed=1 if precond == femgpu.PC_CHEBYSHEV else 2)
    ops = [t[4] for t in inst]
    bs = [t[3] for t in inst]
    xs = [np.zeros_like(b) for b in bs]
    cfg = femgpu.SolverConfig(rtol=1e-8, max_iter=5000, precision=femgpu.FP32_IR, check_interval=5)
    ok, res = femgpu.batch_pcg(ops, bs, xs, cfg, precond)
    assert ok
    iters = set()
    for (mesh, mask, kq, b, op), x, r in zip(inst, xs, res):
        assert r.converged and r.true_residual <= 1e-8, (mesh.nx, mesh.p, r)
        x_ref, _ = O.pcg(mesh, O.Coef(O.DIFF, kappa_q=kq), mask, b, precond=1, rtol=1e-13, max_iter=20000)
        assert np.linalg.norm(x - x_ref) <= 1e-7 * np.linalg.norm(x_ref)
        x1 = np.zeros_like(b)
        r1 = op.pcg(b, x1, cfg, precond)
        assert abs(r1.iterations - r.iterations) <= 2, (r1.iterations, r.iterations)
        iters.add(r.iterations)
    assert len(iters) > 3  # instances converged at different iterations (masks exercised)


def test_batched_zero_rhs_and_mixed_formats():
    need_gpu()
    inst = make_instances([(5, 2), (6, 1), (4, 3)], seed=3)
    ops = [t[4] for t in inst]
    ops[1].set_qdata_format(femgpu.QDATA_AFFINE)
    bs = [t[3] for t in inst]
    bs[2] = np.zeros_like(bs[2])
    xs = [np.zeros_like(b) for b in bs]
    cfg = femgpu.SolverConfig(rtol=1e-8, max_iter=5000, precision=femgpu.FP32_IR)
    ok, res = femgpu.batch_pcg(ops, bs, xs, cfg, femgpu.PC_CHEBYSHEV)
    assert ok
    assert res[2].converged and res[2].iterations == 0 and not xs[2].any()
    for (mesh, mask, kq, b, op), x, r in list(zip(inst, xs, res))[:2]:
        x_ref, _ = O.pcg(mesh, O.Coef(O.DIFF, kappa_q=kq), mask, b, precond=1, rtol=1e-13, max_iter=20000)
        assert r.true_residual <= 1e-8
        assert np.linalg.norm(x - x_ref) <= 1e-7 * np.linalg.norm(x_ref)


def test_batched_rejects_fp64_and_duplicates():
    need_gpu()
    op = femgpu.PADiffusionOperator((3, 3, 3), 1)
    b = np.ones(op.n_dofs())
    with pytest.raises(femgpu.SolverError):
        femgpu.batch_pcg([op], [b], [np.zeros_like(b)], femgpu.SolverConfig(precision=femgpu.FP64))
    with pytest.raises(femgpu.SolverError):
        femgpu.batch_pcg([op, op], [b, b], [np.zeros_like(b), np.zeros_like(b)],
                         femgpu.SolverConfig(precision=femgpu.FP32_IR))
