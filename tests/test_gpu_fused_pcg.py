"""The Jacobi-PCG (and operator-CG) iteration's vector work as one
cooperative launch per iteration (k_pcg_fused_jacobi: p.Ap, the x / r / z
update with r.r and r.z, the stopping test and the direction update, with two
bounded grid barriers) against the three separate kernels (FG_FUSED_PCG=0):
the same block-order sums, so iterations, residuals and solutions are
identical bit for bit, with and without CUDA-graph replay."""
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


def _solve(monkeypatch, fused, graphs, n, p, kq, b, precond, cfg):
    monkeypatch.setenv("FG_FUSED_PCG", "1" if fused else "0")
    monkeypatch.setenv("FG_SOLVER_GRAPHS", "1" if graphs else "0")
    op = femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
    x = np.zeros(op.n_dofs())
    r = op.pcg(b, x, cfg, precond)
    op.close()
    return r, x


@pytest.mark.parametrize("p,n", [(1, 24), (2, 12), (3, 8)])
@pytest.mark.parametrize("precond", [femgpu.PC_JACOBI, femgpu.PC_NONE])
def test_fused_iteration_is_bit_identical(monkeypatch, p, n, precond):
    need_gpu()
    kq = lognormal_kappa_q(n, n, n, p, seed=p)
    mesh = O.Mesh(n, n, n, p)
    b = O.source(mesh, O.ess_mask(mesh)) + 0.0
    b[O.ess_mask(mesh) == 0] += np.random.default_rng(p).standard_normal(int((O.ess_mask(mesh) == 0).sum()))
    cfg = femgpu.SolverConfig(rtol=1e-10, max_iter=5000)
    ref, x_ref = _solve(monkeypatch, False, True, n, p, kq, b, precond, cfg)
    assert ref.converged and ref.iterations > 20
    for graphs in (True, False):
        r, x = _solve(monkeypatch, True, graphs, n, p, kq, b, precond, cfg)
        assert r.converged and r.iterations == ref.iterations
        assert r.final_residual == ref.final_residual and r.true_residual == ref.true_residual
        assert np.array_equal(x, x_ref)
    # the iteration cap ends the fused loop exactly where the separate kernels end
    cap = femgpu.SolverConfig(rtol=1e-14, max_iter=7)
    a, xa = _solve(monkeypatch, False, True, n, p, kq, b, precond, cap)
    f, xf = _solve(monkeypatch, True, True, n, p, kq, b, precond, cap)
    assert not a.converged and not f.converged and np.array_equal(xa, xf)
