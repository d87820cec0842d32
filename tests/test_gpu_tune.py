"""Tile shapes and the batched autotuner.

fg_op_set_tile re-lays out the quadrature data for items of TZ element
layers: every apply form must keep the oracle tolerances (FP64 1e-12
relative, FP32 2e-5) for any TZ, including depths that do not divide nz.
fg_batch_autotune times each candidate on the batched FP32 apply, leaves the
fastest on the operators, and the batched solves that follow still reach the
FP64 target with the same answers as before tuning (<= 1e-7 relative).
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


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def f32_apply(op, x):
    x32 = np.ascontiguousarray(x, dtype=np.float32)
    y32 = np.zeros_like(x32)
    rc = femgpu.lib().fg_op_apply_f32(op.handle, x32.ctypes.data, y32.ctypes.data, 0, 1, femgpu.HOST)
    assert rc == 0, femgpu.last_error()
    return y32.astype(np.float64)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_set_tile_keeps_every_apply_form(p):
    need_gpu()
    nx, ny, nz = (37, 9, 13) if p < 3 else (33, 5, 7)
    kq = lognormal_kappa_q(nx, ny, nz, p, seed=p)
    mesh = O.Mesh(nx, ny, nz, p)
    mask = O.ess_mask(mesh)
    coef = O.Coef(O.DIFF, kappa_q=kq)
    x = np.random.default_rng(p).standard_normal(mesh.ndofs)
    ref = O.apply_constrained(mesh, coef, mask, x)
    op = femgpu.PADiffusionOperator((nx, ny, nz), p, kappa=kq)
    y0 = op.matvec(x, constrained=True)
    tz0 = op.tile[2]
    for tz in (1, 2, 3, 4, 16, tz0):
        op.set_tile(tz)
        assert op.tile[2] == tz
        y = op.matvec(x, constrained=True)
        assert rel(y, ref) <= 1e-12 and rel(y, y0) <= 1e-13
        assert rel(f32_apply(op, x), ref) <= 2e-5
    # affine format rebuilt for the new layout
    op.set_qdata_format(femgpu.QDATA_AFFINE)
    op.set_tile(2)
    assert rel(op.matvec(x, constrained=True), ref) <= 1e-12
    assert rel(f32_apply(op, x), ref) <= 2e-5
    with pytest.raises(femgpu.SolverError):
        op.set_tile(0)


def test_autotune_then_batch_solve():
    need_gpu()
    rng = np.random.default_rng(11)
    ops, bs, singles = [], [], []
    cfg = femgpu.SolverConfig(rtol=1e-8, max_iter=5000, precision=femgpu.FP32_IR, check_interval=5)
    for i in range(10):
        n, p = int(rng.integers(6, 21)), int(rng.integers(1, 4))
        kq = lognormal_kappa_q(n, n, n, p, seed=300 + i)
        op = femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
        b = rng.standard_normal(op.n_dofs())
        b.reshape(op.NK, op.NJ, op.NI)[[0, -1]] = 0.0
        b.reshape(op.NK, op.NJ, op.NI)[:, [0, -1]] = 0.0
        b.reshape(op.NK, op.NJ, op.NI)[:, :, [0, -1]] = 0.0
        x = np.zeros_like(b)
        r = op.pcg(b, x, cfg, femgpu.PC_CHEBYSHEV)
        assert r.converged
        ops.append(op)
        bs.append(b)
        singles.append(x)
    table = femgpu.batch_autotune(ops, reps=3)
    assert sum(e["instances"] for e in table) == len(ops)
    for e in table:
        tried = {tz: t for tz, t in e["us"].items() if t is not None}
        other = [t for t in e["us_other"].items() if t[1] is not None]
        assert e["tz"] in tried and tried[e["tz"]] == min(tried.values())
        assert not other or tried[e["tz"]] <= min(t for _, t in other)
        assert e["format"] in (femgpu.QDATA_FULL, femgpu.QDATA_AFFINE)
        assert other  # box meshes: both formats were timed
    for op in ops:
        assert op.tile[2] in femgpu.TUNE_TZ
    xs = [np.zeros_like(b) for b in bs]
    ok, res = femgpu.batch_pcg(ops, bs, xs, cfg, femgpu.PC_CHEBYSHEV)
    assert ok
    for x, xs1, r in zip(xs, singles, res):
        assert r.true_residual <= 1e-8
        assert rel(x, xs1) <= 1e-7


def test_autotune_keeps_full_format_when_a_member_is_not_affine():
    """A class with one distorted mesh (a moved interior vertex): the affine
    candidate is refused for the whole class, the tuner keeps the full format
    there and the batched solve still matches the single solves; an all-box
    class of another order may still move to the affine format."""
    need_gpu()
    rng = np.random.default_rng(5)
    cfg = femgpu.SolverConfig(rtol=1e-8, max_iter=5000, precision=femgpu.FP32_IR, check_interval=5)
    ops, bs, singles = [], [], []
    for i, (n, p, distort) in enumerate([(8, 2, False), (9, 2, True), (10, 1, False), (7, 1, False)]):
        mesh = (n, n, n)
        if distort:
            k, j, ii = np.meshgrid(np.arange(n + 1), np.arange(n + 1), np.arange(n + 1), indexing="ij")
            v = np.stack([ii / n, j / n, k / n], axis=-1).astype(np.float64)
            v[n // 2, n // 2, n // 2] += 0.3 / n
            mesh = dict(nx=n, ny=n, nz=n, vcoord=v.reshape(-1, 3))
        op = femgpu.PADiffusionOperator(mesh, p, kappa=lognormal_kappa_q(n, n, n, p, seed=500 + i))
        b = rng.standard_normal(op.n_dofs())
        b3 = b.reshape(op.NK, op.NJ, op.NI)
        b3[[0, -1]], b3[:, [0, -1]], b3[:, :, [0, -1]] = 0.0, 0.0, 0.0
        x = np.zeros_like(b)
        assert op.pcg(b, x, cfg, femgpu.PC_CHEBYSHEV).converged
        ops.append(op)
        bs.append(b)
        singles.append(x)
    table = femgpu.batch_autotune(ops, reps=2)
    q2 = [e for e in table if e["order"] == 2]
    assert len(q2) == 1 and q2[0]["format"] == femgpu.QDATA_FULL
    assert all(t is None for t in q2[0]["us_other"].values())
    q1 = [e for e in table if e["order"] == 1]
    assert q1 and all(any(t is not None for t in e["us_other"].values()) for e in q1)
    xs = [np.zeros_like(b) for b in bs]
    ok, res = femgpu.batch_pcg(ops, bs, xs, cfg, femgpu.PC_CHEBYSHEV)
    assert ok
    for x, x1, r in zip(xs, singles, res):
        assert r.true_residual <= 1e-8
        assert rel(x, x1) <= 1e-7
    for op in ops:
        op.close()
