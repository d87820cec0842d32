"""Solver chunks replayed as CUDA graphs perform exactly the launches of the
direct chunks: solutions are bitwise identical and iteration counts equal
with graphs on and off (FG_SOLVER_GRAPHS=0, read when a handle is created),
for every solver loop (PCG-Jacobi, PCG-Chebyshev, mixed precision, learned
flexible CG).  The learned correction computed on a side stream beside the
smoother (default) equals the in-line order (FG_NN_OVERLAP=0) bit for bit."""
import os

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


def _op(n, p, kq, graphs, overlap=True):
    env = {"FG_SOLVER_GRAPHS": "1" if graphs else "0", "FG_NN_OVERLAP": "1" if overlap else "0"}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


@pytest.mark.parametrize("precond,precision", [(femgpu.PC_JACOBI, femgpu.FP64),
                                               (femgpu.PC_CHEBYSHEV, femgpu.FP64),
                                               (femgpu.PC_CHEBYSHEV, femgpu.FP32_IR),
                                               (femgpu.PC_JACOBI, femgpu.FP32_IR)])
def test_graph_replay_is_bitwise_identical(precond, precision):
    need_gpu()
    n, p = 12, 2
    kq = lognormal_kappa_q(n, n, n, p, seed=3)
    mesh = O.Mesh(n, n, n, p)
    mask = O.ess_mask(mesh)
    b = np.random.default_rng(4).standard_normal(mesh.ndofs)
    b[mask == 1] = 0.0
    xs, its = [], []
    for graphs in (True, False):
        op = _op(n, p, kq, graphs)
        x = np.zeros(mesh.ndofs)
        cfg = femgpu.SolverConfig(rtol=1e-10, max_iter=5000, precision=precision, check_interval=3)
        r = op.pcg(b, x, cfg, precond)
        assert r.converged
        xs.append(x)
        its.append(r.iterations)
        op.close()
    assert its[0] == its[1]
    assert np.array_equal(xs[0], xs[1])


@pytest.mark.parametrize("precision", [femgpu.FP64, femgpu.FP32_IR])
def test_graph_replay_learned_fcg(precision):
    need_gpu()
    n = 16
    kq = lognormal_kappa_q(n, n, n, 1, seed=5)
    mesh = O.Mesh(n, n, n, 1)
    mask = O.ess_mask(mesh)
    b = np.random.default_rng(6).standard_normal(mesh.ndofs)
    b[mask == 1] = 0.0
    net = femgpu.UNet(seed=2)
    xs, its = [], []
    # graphs + network beside the smoother, direct launches, network in line
    for graphs, overlap in ((True, True), (False, True), (True, False)):
        op = _op(n, 1, kq, graphs, overlap)
        femgpu.set_nodal_kappa(op, femgpu.nodal_kappa_from_q(kq, n, n, n), 1)
        femgpu.attach_unet(op, net)
        x = np.zeros(mesh.ndofs)
        cfg = femgpu.SolverConfig(rtol=1e-9, max_iter=2000, precision=precision, check_interval=2)
        r = op.pcg(b, x, cfg, femgpu.PC_CHEB_NN)
        assert r.converged and r.true_residual <= 1e-9
        xs.append(x)
        its.append(r.iterations)
        op.close()
    assert its[0] == its[1] == its[2]
    assert np.array_equal(xs[0], xs[1]) and np.array_equal(xs[0], xs[2])
