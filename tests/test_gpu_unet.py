"""Learned coarse correction: the BF16 U-net's forward pass and hand-written
backward pass against the NumPy reference (oracle/unet_ref.py), training by
the library's own kernels, and its use inside flexible CG.

Tolerances (BF16 storage, FP32 accumulation in a different order than the
reference): forward output 2e-2 relative (2-norm), loss 1e-2 relative, every
layer's weight and bias gradient 5e-2 relative (2-norm).  The solves keep
the FP64 targets: true relative residual <= 1e-8, error vs the oracle <= 1e-7.
"""
import numpy as np
import pytest

from conftest import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import femgpu  # noqa: E402
import unet_ref as R  # noqa: E402  (oracle/unet_ref.py)
from femgpu.fields import lognormal_kappa_q  # noqa: E402


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-30)


def test_forward_matches_reference():
    need_gpu()
    net = femgpu.UNet(seed=3)
    rng = np.random.default_rng(0)
    inp = rng.standard_normal((2, 9, 13, 9, 2)).astype(np.float32)
    out = net.forward(inp)
    ref = R.forward(net.get_params(), inp)["out"][..., 0]
    assert out.shape == (2, 9, 13, 9)
    assert rel(out, ref) <= 2e-2, rel(out, ref)


def test_gradients_match_reference():
    need_gpu()
    net = femgpu.UNet(seed=5)
    rng = np.random.default_rng(1)
    inp = rng.standard_normal((2, 9, 9, 13, 2)).astype(np.float32)
    tgt = rng.standard_normal((2, 9, 9, 13)).astype(np.float32)
    loss = net.loss_grad(inp, tgt)
    g = net.get_grads()
    loss_ref, g_ref = R.loss_grad(net.get_params(), inp, tgt)
    assert abs(loss - loss_ref) <= 1e-2 * loss_ref
    o = 0
    for name, (ci, co) in zip(R.LAYERS, R.layer_shapes()):
        nw = co * 27 * ci
        for part, sl in (("W", slice(o, o + nw)), ("b", slice(o + nw, o + nw + co))):
            e = rel(g[sl], g_ref[sl])
            assert e <= 5e-2, (name, part, e)
        o += nw + co


def test_training_reduces_loss():
    need_gpu()
    net = femgpu.UNet(seed=7)
    rng = np.random.default_rng(2)
    inp = rng.standard_normal((4, 9, 9, 9, 2)).astype(np.float32)
    # a smooth function of the input as the regression target
    tgt = inp[..., 0].copy()
    for ax in (1, 2, 3):
        tgt = 0.25 * np.roll(tgt, 1, ax) + 0.5 * tgt + 0.25 * np.roll(tgt, -1, ax)
    l0 = net.loss_grad(inp, tgt)
    for _ in range(60):
        last = net.train_step(inp, tgt, 3e-3)
    assert last < 0.5 * l0, (l0, last)


def _q1_problem(n, seed):
    kq = lognormal_kappa_q(n, n, n, 1, seed=seed)
    mesh = O.Mesh(n, n, n, 1)
    mask = O.ess_mask(mesh)
    rng = np.random.default_rng(seed)
    b = O.pa_apply(mesh, O.Coef(O.MASS), rng.standard_normal(mesh.ndofs))
    b[mask == 1] = 0.0
    op = femgpu.PADiffusionOperator((n, n, n), 1, kappa=kq)
    femgpu.set_nodal_kappa(op, femgpu.nodal_kappa_from_q(kq, n, n, n))
    return mesh, mask, kq, b, op


def test_learned_fcg_trains_solves_and_falls_back():
    need_gpu()
    n = 16
    net = femgpu.UNet(seed=11)
    # pairs from plain Chebyshev-PCG on two training fields
    ins, tgts = [], []
    for seed in (21, 22):
        _, _, _, b, op = _q1_problem(n, seed)
        xi, t = femgpu.collect_pairs(op, b, every=2, max_pairs=20)
        assert xi.shape[1:] == (9, 9, 9, 2) and xi.shape[0] == t.shape[0] >= 5
        ins.append(xi)
        tgts.append(t)
    xin = torch.cat(ins).contiguous()
    tgt = torch.cat(tgts).contiguous()
    l0 = net.loss_grad(xin[:8].contiguous(), tgt[:8].contiguous())
    for it in range(80):
        k = (it * 8) % (xin.shape[0] - 8)
        loss = net.train_step(xin[k:k + 8].contiguous(), tgt[k:k + 8].contiguous(), 2e-3)
    assert loss < l0
    mesh, mask, kq, b, op = _q1_problem(n, 99)  # held out
    x_ref, _ = O.pcg(mesh, O.Coef(O.DIFF, kappa_q=kq), mask, b, precond=1, rtol=1e-13, max_iter=20000)
    femgpu.attach_unet(op, net)
    for prec in (femgpu.FP64, femgpu.FP32_IR):
        x = np.zeros(mesh.ndofs)
        r = op.pcg(b, x, femgpu.SolverConfig(rtol=1e-8, max_iter=2000, precision=prec), femgpu.PC_CHEB_NN)
        assert r.converged and r.true_residual <= 1e-8
        assert rel(x, x_ref) <= 1e-7
    # a budget of 3 iterations forces the fallback to plain Chebyshev-PCG
    x = np.zeros(mesh.ndofs)
    r = op.pcg(b, x, femgpu.SolverConfig(rtol=1e-8, max_iter=2000, nn_budget=3, check_interval=2),
               femgpu.PC_CHEB_NN)
    assert r.converged and r.extra["nn_fallback"] == 1 and r.true_residual <= 1e-8


def test_learned_precond_requires_network():
    need_gpu()
    op = femgpu.PADiffusionOperator((8, 8, 8), 1)
    b = np.ones(op.n_dofs())
    with pytest.raises(femgpu.SolverError):
        op.pcg(b, np.zeros_like(b), femgpu.SolverConfig(), femgpu.PC_CHEB_NN)
    with pytest.raises(femgpu.SolverError):
        femgpu.set_nodal_kappa(femgpu.PADiffusionOperator((6, 8, 8), 1), np.ones(7 * 9 * 9))
