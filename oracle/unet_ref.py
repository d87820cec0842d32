"""NumPy reference of the learned-correction U-net (TEST INFRASTRUCTURE ONLY).

Used by tests/ to check the GPU forward pass and the hand-written backward
pass (loss and every parameter gradient).  The network has no counterpart in
the fem-rs reference; this file restates the architecture documented in
fem-rs_b200/csrc/unet_host.cuh and rounds to BF16 at the same points the GPU
kernels store BF16 (inputs, weights, activations, activation gradients);
sums are carried in float64.

Parameter layout (as fg_unet_get_params): per layer W[cout][27][cin] with
tap = (dz+1)*9 + (dy+1)*3 + (dx+1), then b[cout]; layers l0a, l0b, l1a, l1b,
l2a, l2b, l1c, l0c, out.
"""
from __future__ import annotations

import numpy as np

LAYERS = ["l0a", "l0b", "l1a", "l1b", "l2a", "l2b", "l1c", "l0c", "out"]


def bf16(x):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def layer_shapes(c0=16, c1=32, c2=48):
    cin = [2, c0, c0, c1, c1, c2, c2 + c1, c1 + c0, c0]
    cout = [c0, c0, c1, c1, c2, c2, c1, c0, 8]
    return list(zip(cin, cout))


def unpack(params, c=(16, 32, 48)):
    out, o = {}, 0
    for name, (ci, co) in zip(LAYERS, layer_shapes(*c)):
        nw = co * 27 * ci
        out[name] = (params[o:o + nw].reshape(co, 27, ci).astype(np.float64), params[o + nw:o + nw + co].astype(np.float64))
        o += nw + co
    assert o == len(params)
    return out


def pack(grads, c=(16, 32, 48)):
    return np.concatenate([np.concatenate([grads[n][0].ravel(), grads[n][1].ravel()]) for n in LAYERS])


def _shift(x, dz, dy, dx):
    """y[v] = x[v + d] with zero outside (x: [B,Z,Y,X,C])."""
    B, Z, Y, X, C = x.shape
    y = np.zeros_like(x)
    zs, ze = max(0, -dz), min(Z, Z - dz)
    ys, ye = max(0, -dy), min(Y, Y - dy)
    xs, xe = max(0, -dx), min(X, X - dx)
    y[:, zs:ze, ys:ye, xs:xe] = x[:, zs + dz:ze + dz, ys + dy:ye + dy, xs + dx:xe + dx]
    return y


def taps():
    return [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]


def conv(x, W, b):
    out = np.zeros(x.shape[:4] + (W.shape[0],))
    for t, (dz, dy, dx) in enumerate(taps()):
        out += _shift(x, dz, dy, dx) @ W[:, t, :].T
    return out + b


def conv_bwd(x, W, dy_):
    """(dW, db, dx) of out = conv(x, W, b) given d(out)."""
    dW = np.zeros_like(W)
    dx = np.zeros_like(x)
    flat = dy_.reshape(-1, dy_.shape[-1])
    for t, (dz, dy, dxx) in enumerate(taps()):
        xs = _shift(x, dz, dy, dxx).reshape(-1, x.shape[-1])
        dW[:, t, :] = flat.T @ xs
        dx += _shift(dy_ @ W[:, t, :], -dz, -dy, -dxx)
    return dW, flat.sum(axis=0), dx


def hat_weights(parity):
    return [(0, 1.0)] if parity == 0 else [(0, 0.5), (1, 0.5)]


def prolong(xc, shape_f):
    B, Zf, Yf, Xf = shape_f
    C = xc.shape[-1]
    out = np.zeros((B, Zf, Yf, Xf, C))
    for z in range(Zf):
        for y in range(Yf):
            for x in range(Xf):
                s = 0.0
                for a, wa in hat_weights(z & 1):
                    for bb, wb in hat_weights(y & 1):
                        for d, wd in hat_weights(x & 1):
                            s = s + wa * wb * wd * xc[:, (z >> 1) + a, (y >> 1) + bb, (x >> 1) + d]
                out[:, z, y, x] = s
    return out


def restrict(xf):
    B, Zf, Yf, Xf, C = xf.shape
    Zc, Yc, Xc = (Zf + 1) // 2, (Yf + 1) // 2, (Xf + 1) // 2
    out = np.zeros((B, Zc, Yc, Xc, C))
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                w = (0.5 if dz else 1.0) * (0.5 if dy else 1.0) * (0.5 if dx else 1.0) * 0.125
                for z in range(Zc):
                    fz = 2 * z + dz
                    if fz < 0 or fz >= Zf:
                        continue
                    for y in range(Yc):
                        fy = 2 * y + dy
                        if fy < 0 or fy >= Yf:
                            continue
                        for x in range(Xc):
                            fx = 2 * x + dx
                            if fx < 0 or fx >= Xf:
                                continue
                            out[:, z, y, x] += w * xf[:, fz, fy, fx]
    return out


def forward(params, inp, c=(16, 32, 48)):
    """inp [B,Z,Y,X,2] -> dict of BF16-rounded activations; 'out' [B,Z,Y,X,8]."""
    P = unpack(params, c)
    W = {k: (bf16(v[0]), v[1]) for k, v in P.items()}
    relu = lambda a: np.maximum(a, 0.0)
    A = {"x0": bf16(inp)}
    A["a0"] = bf16(relu(conv(A["x0"], *W["l0a"])))
    A["h0"] = bf16(relu(conv(A["a0"], *W["l0b"])))
    A["x1"] = bf16(restrict(A["h0"]))
    A["a1"] = bf16(relu(conv(A["x1"], *W["l1a"])))
    A["h1"] = bf16(relu(conv(A["a1"], *W["l1b"])))
    A["x2"] = bf16(restrict(A["h1"]))
    A["a2"] = bf16(relu(conv(A["x2"], *W["l2a"])))
    A["h2"] = bf16(relu(conv(A["a2"], *W["l2b"])))
    A["u1"] = bf16(prolong(A["h2"], A["h1"].shape[:4]))
    A["cat1"] = np.concatenate([A["u1"], A["h1"]], axis=-1)
    A["g1"] = bf16(relu(conv(A["cat1"], *W["l1c"])))
    A["u0"] = bf16(prolong(A["g1"], A["h0"].shape[:4]))
    A["cat0"] = np.concatenate([A["u0"], A["h0"]], axis=-1)
    A["g0"] = bf16(relu(conv(A["cat0"], *W["l0c"])))
    A["out"] = bf16(conv(A["g0"], *W["out"]))
    A["W"] = W
    return A


def loss_grad(params, inp, target, c=(16, 32, 48)):
    """(loss, flat gradient) of mean((out[...,0] - target)^2)."""
    A = forward(params, inp, c)
    nv = target.size
    d = A["out"][..., 0] - target
    loss = float((d * d).sum() / nv)
    dout = np.zeros_like(A["out"])
    dout[..., 0] = bf16(2.0 * d / nv)
    return loss, backward(A, dout, c)


def backward(A, dout, c=(16, 32, 48)):
    """Flat parameter gradient from the activations A of forward() and the
    (BF16-rounded) output gradient dout [B,Z,Y,X,8]."""
    W = A["W"]
    g = {}
    c0, c1, c2 = c
    mask = lambda a: (a > 0).astype(np.float64)
    g["out"] = conv_bwd(A["g0"], W["out"][0], dout)[:2]
    dg0 = bf16(conv_bwd(A["g0"], W["out"][0], dout)[2]) * mask(A["g0"])
    dW, db, dcat0 = conv_bwd(A["cat0"], W["l0c"][0], dg0)
    g["l0c"] = (dW, db)
    dcat0 = bf16(dcat0)
    dg1 = bf16(8.0 * restrict(dcat0[..., :c1])) * mask(A["g1"])
    dW, db, dcat1 = conv_bwd(A["cat1"], W["l1c"][0], dg1)
    g["l1c"] = (dW, db)
    dcat1 = bf16(dcat1)
    dh2 = bf16(8.0 * restrict(dcat1[..., :c2])) * mask(A["h2"])
    dW, db, da2 = conv_bwd(A["a2"], W["l2b"][0], dh2)
    g["l2b"] = (dW, db)
    da2 = bf16(da2) * mask(A["a2"])
    dW, db, dx2 = conv_bwd(A["x2"], W["l2a"][0], da2)
    g["l2a"] = (dW, db)
    dx2 = bf16(dx2)
    dh1 = bf16(dcat1[..., c2:] + 0.125 * prolong(dx2, A["h1"].shape[:4])) * mask(A["h1"])
    dW, db, da1 = conv_bwd(A["a1"], W["l1b"][0], dh1)
    g["l1b"] = (dW, db)
    da1 = bf16(da1) * mask(A["a1"])
    dW, db, dx1 = conv_bwd(A["x1"], W["l1a"][0], da1)
    g["l1a"] = (dW, db)
    dx1 = bf16(dx1)
    dh0 = bf16(dcat0[..., c1:] + 0.125 * prolong(dx1, A["h0"].shape[:4])) * mask(A["h0"])
    dW, db, da0 = conv_bwd(A["a0"], W["l0b"][0], dh0)
    g["l0b"] = (dW, db)
    da0 = bf16(da0) * mask(A["a0"])
    dW, db, _ = conv_bwd(A["x0"], W["l0a"][0], da0)
    g["l0a"] = (dW, db)
    return pack(g, c)
