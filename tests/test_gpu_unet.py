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


@pytest.mark.parametrize("channels,shape,grads", [
    ((16, 32, 48), (2, 9, 13, 9), True),
    ((16, 32, 48), (1, 33, 33, 33), True),   # the network volume of the 128^3 Q2 learned solve
    ((16, 64, 16), (1, 17, 13, 9), True),    # 64 output channels
    ((32, 48, 64), (1, 17, 13, 9), False),   # 112 input channels (its backward needs a 112-channel
                                             # input gradient, which neither path supports)
    ((8, 16, 32), (3, 9, 9, 13), False),     # 24-channel input (K padded to 32; its backward needs a
                                             # 24-channel input gradient, which mma.sync does not support)
    ((8, 8, 8), (2, 13, 9, 9), True),        # 8-channel layers (K padded to 16)
])
def test_tcgen05_convolutions_match_mma_sync(channels, shape, grads, monkeypatch):
    """The convolutions on tcgen05 (TMEM accumulators; FG_UNET_TC=1) against
    the mma.sync kernels (the default) on the same weights and input: the
    forward output, the loss and every layer's weight and bias gradient (the
    input gradients run the same convolution with flipped weights).  Both
    accumulate BF16 products in FP32, in different orders, so they agree to
    BF16 rounding: 1e-2 relative for the output and loss, 5e-2 for the
    gradients, the tolerances used against the reference above."""
    need_gpu()
    rng = np.random.default_rng(7)
    inp = rng.standard_normal(shape + (2,)).astype(np.float32)
    tgt = rng.standard_normal(shape).astype(np.float32)
    monkeypatch.setenv("FG_UNET_TC", "0")
    legacy = femgpu.UNet(channels=channels, seed=11)
    monkeypatch.setenv("FG_UNET_TC", "1")
    tc = femgpu.UNet(channels=channels, seed=11)
    out_l, out_t = legacy.forward(inp), tc.forward(inp)
    assert np.all(np.isfinite(out_t))
    assert rel(out_t, out_l) <= 1e-2, rel(out_t, out_l)
    if not grads:
        return
    loss_l, loss_t = legacy.loss_grad(inp, tgt), tc.loss_grad(inp, tgt)
    assert abs(loss_t - loss_l) <= 1e-2 * abs(loss_l), (loss_t, loss_l)
    g_l, g_t = legacy.get_grads(), tc.get_grads()
    assert g_l.shape == g_t.shape
    c0, c1, c2 = channels
    shapes = [(2, c0), (c0, c0), (c0, c1), (c1, c1), (c1, c2), (c2, c2), (c2 + c1, c1), (c1 + c0, c0), (c0, 8)]
    o = 0
    for li, (ci, co) in enumerate(shapes):
        nw = co * 27 * ci
        for part, sl in (("W", slice(o, o + nw)), ("b", slice(o + nw, o + nw + co))):
            e = rel(g_t[sl], g_l[sl])
            assert e <= 5e-2, (li, part, e)
        o += nw + co
    assert o == g_t.size


def _q1_problem(n, seed, p=1):
    kq = lognormal_kappa_q(n, n, n, p, seed=seed)
    mesh = O.Mesh(n, n, n, p)
    mask = O.ess_mask(mesh)
    rng = np.random.default_rng(seed)
    b = O.pa_apply(mesh, O.Coef(O.MASS), rng.standard_normal(mesh.ndofs))
    b[mask == 1] = 0.0
    op = femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
    femgpu.set_nodal_kappa(op, femgpu.nodal_kappa_from_q(kq, n, n, n, p))
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
    # cost-aware choice: with an expected iteration ratio no network could
    # meet, the solver measures both iteration costs and runs plain
    # Chebyshev-PCG from the start (same iterations as the plain solve); with a
    # tiny ratio it starts with the network (which this small test network may
    # still drop at the iteration budget: fallback 1)
    x = np.zeros(mesh.ndofs)
    plain = op.pcg(b, x, femgpu.SolverConfig(rtol=1e-8, max_iter=2000), femgpu.PC_CHEBYSHEV)
    for prec in (femgpu.FP64, femgpu.FP32_IR):
        x = np.zeros(mesh.ndofs)
        r = op.pcg(b, x, femgpu.SolverConfig(rtol=1e-8, max_iter=2000, precision=prec, nn_budget=plain.iterations,
                                             nn_iter_ratio=5.0), femgpu.PC_CHEB_NN)
        assert r.converged and r.extra["nn_fallback"] == 2 and r.true_residual <= 1e-8
        if prec == femgpu.FP64:
            assert r.iterations == plain.iterations
        x = np.zeros(mesh.ndofs)
        r = op.pcg(b, x, femgpu.SolverConfig(rtol=1e-8, max_iter=2000, precision=prec, nn_budget=plain.iterations,
                                             nn_iter_ratio=1e-3), femgpu.PC_CHEB_NN)
        assert r.converged and r.extra["nn_fallback"] != 2 and r.true_residual <= 1e-8


def _restrict_levels(v, shape, levels):
    """R^L of a plain-layout vertex field, rounded to FP32 after each level."""
    a = np.asarray(v, dtype=np.float64).reshape((1,) + shape + (1,))
    for _ in range(levels):
        a = R.restrict(a).astype(np.float32).astype(np.float64)
    return a[0, ..., 0]


@pytest.mark.parametrize("p,levels", [(1, 1), (1, 2), (2, 2)])
def test_energy_loss_gradients_match_reference(p, levels):
    """fg_unet_train_energy: loss (c.Ac/2 - c.r)/(s^2 64^L Nc), c = s 8^L P^L n,
    and every parameter gradient against the NumPy network with the oracle's
    constrained apply."""
    need_gpu()
    n, B = 16 // p, 2
    mesh, mask, kq, _, op = _q1_problem(n, 31, p)
    kn = femgpu.nodal_kappa_from_q(kq, n, n, n, p)
    femgpu.set_nodal_kappa(op, kn, levels)
    shape = (p * n + 1,) * 3
    Vc = femgpu.nn_volume(op)
    assert Vc == ((p * n >> levels) + 1,) * 3
    rng = np.random.default_rng(32)
    res = rng.standard_normal((B, mesh.ndofs))
    res[:, mask == 1] = 0.0
    dres = torch.tensor(np.stack([op.to_native(r) for r in res]), device="cuda")
    net = femgpu.UNet(seed=13)
    params = net.get_params()
    loss = net.train_energy(op, dres, 0.0)
    g = net.get_grads()
    # reference
    lk = _restrict_levels(np.log(kn), shape, levels).astype(np.float32)
    nv = int(np.prod(Vc))
    inp = np.zeros((B,) + Vc + (2,), dtype=np.float32)
    scales = []
    for b in range(B):
        rc = _restrict_levels(res[b], shape, levels).astype(np.float32)
        s = float(np.sqrt(np.mean(rc.astype(np.float64) ** 2)))
        scales.append(s)
        inp[b, ..., 0] = (rc / s).astype(np.float32)
        inp[b, ..., 1] = lk
    A = R.forward(params, inp)
    coef = 1.0 / (nv * B)
    mult = 8.0 ** levels
    dout = np.zeros_like(A["out"])
    loss_ref = 0.0
    coefq = O.Coef(O.DIFF, kappa_q=kq)
    for b in range(B):
        c = A["out"][b:b + 1, ..., :1]
        for _ in range(levels):
            c = R.prolong(c, (1,) + tuple(2 * d - 1 for d in c.shape[1:4]))
        c = scales[b] * mult * c[0, ..., 0].ravel()
        c[mask == 1] = 0.0
        ac = O.apply_constrained(mesh, coefq, mask, c)
        loss_ref += (0.5 * c @ ac - c @ res[b]) / (scales[b] ** 2 * mult ** 2 * nv) / B
        gc = _restrict_levels(ac - res[b], shape, levels)
        dout[b, ..., 0] = R.bf16(coef / scales[b] * gc)
    g_ref = R.backward(A, dout)
    assert abs(loss - loss_ref) <= 1e-2 * abs(loss_ref) + 1e-6, (loss, loss_ref)
    o = 0
    for name, (ci, co) in zip(R.LAYERS, R.layer_shapes()):
        nw = co * 27 * ci
        for part, sl in (("W", slice(o, o + nw)), ("b", slice(o + nw, o + nw + co))):
            e = rel(g[sl], g_ref[sl])
            assert e <= 5e-2, (name, part, e)
        o += nw + co


def test_energy_training_reduces_loss_and_helps_fcg():
    """Energy-loss training on residuals of plain Chebyshev-PCG: the loss
    falls, and flexible CG with the trained two-level correction converges to
    the FP64 target on a held-out coefficient field."""
    need_gpu()
    n = 32
    net = femgpu.UNet(seed=17)
    fields = []
    for seed in (41, 42):
        mesh, mask, kq, b, op = _q1_problem(n, seed)
        femgpu.set_nodal_kappa(op, femgpu.nodal_kappa_from_q(kq, n, n, n), 2)
        fields.append((op, femgpu.collect_residuals(op, b, every=2, max_res=24)))
    assert all(r.shape[0] >= 8 for _, r in fields)
    first = [net.train_energy(op, r[:8].contiguous(), 0.0) for op, r in fields]
    for it in range(60):
        op, r = fields[it % 2]
        k = (it * 4) % (r.shape[0] - 4)
        net.train_energy(op, r[k:k + 4].contiguous(), 2e-3)
    last = [net.train_energy(op, r[:8].contiguous(), 0.0) for op, r in fields]
    # the loss is negative at a useful correction (energy decrease)
    assert sum(last) < sum(first) and sum(last) < 0.0, (first, last)
    mesh, mask, kq, b, op = _q1_problem(n, 98)
    femgpu.set_nodal_kappa(op, femgpu.nodal_kappa_from_q(kq, n, n, n), 2)
    femgpu.attach_unet(op, net)
    x = np.zeros(mesh.ndofs)
    r = op.pcg(b, x, femgpu.SolverConfig(rtol=1e-8, max_iter=2000), femgpu.PC_CHEB_NN)
    assert r.converged and r.true_residual <= 1e-8


def test_learned_precond_requires_network():
    need_gpu()
    op = femgpu.PADiffusionOperator((8, 8, 8), 1)
    b = np.ones(op.n_dofs())
    with pytest.raises(femgpu.SolverError):
        op.pcg(b, np.zeros_like(b), femgpu.SolverConfig(), femgpu.PC_CHEB_NN)
    with pytest.raises(femgpu.SolverError):
        femgpu.set_nodal_kappa(femgpu.PADiffusionOperator((6, 8, 8), 1), np.ones(7 * 9 * 9))
    with pytest.raises(femgpu.SolverError):
        femgpu.set_nodal_kappa(femgpu.PADiffusionOperator((8, 8, 8), 1), np.ones(9 * 9 * 9), 2)
    with pytest.raises(femgpu.SolverError):
        femgpu.set_nodal_kappa(femgpu.PADiffusionOperator((16, 16, 16), 1), np.ones(17 ** 3), 5)
