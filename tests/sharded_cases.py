"""Shared cases of the sharded-operator tests: a perturbed hex box with
lognormal kappa, the oracle's whole-mesh answers, and the comparison of the
ranks' assembled pieces with them."""
import numpy as np

import oracle as O


def problem(nx=5, ny=4, nz=7, p=2, seed=3):
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    vc = np.stack([i / nx, j / ny, k / nz], axis=-1).reshape(-1, 3).astype(np.float64)
    inner = ((i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)).reshape(-1, 1)
    h = np.array([1.0 / nx, 1.0 / ny, 1.0 / nz])
    vc += 0.2 * h * rng.uniform(-1, 1, size=vc.shape) * inner  # well-shaped elements at any size
    kq = np.exp(rng.normal(size=nx * ny * nz * (p + 1) ** 3))
    return dict(nx=nx, ny=ny, nz=nz, vcoord=vc), p, kq


def reference(mesh, p, kq, tags):
    m = O.Mesh(mesh["nx"], mesh["ny"], mesh["nz"], p, vcoord=mesh["vcoord"])
    coef = O.Coef(O.DIFF, kappa_q=kq)
    ess = O.ess_mask(m, tags)
    x = np.random.default_rng(11).normal(size=m.ndofs)
    b = O.source(m, ess)
    xs, info = O.pcg(m, coef, ess, b, precond=1, rtol=1e-10, max_iter=2000)
    return dict(x=x, b=b, y=O.apply_constrained(m, coef, ess, x), d=O.diagonal(m, coef, ess), xs=xs,
                it=info["iterations"], shape=m.shape)


def check(results, ref, tol_apply=1e-13):
    results = sorted(results, key=lambda r: r["rank"])
    NK, NJ, NI = ref["shape"]
    for key, want, tol in (("y", ref["y"], tol_apply), ("d", ref["d"], tol_apply), ("x", ref["xs"], 1e-7)):
        got = np.concatenate([r[key] for r in results])
        assert got.shape == want.shape
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err <= tol, (key, err)
    yg = ref["y"].reshape(NK, NJ, NI)
    for r in results:  # both copies of every interface plane hold the assembled value
        yl = r["y_local"].reshape(r["NK"], NJ, NI)
        np.testing.assert_allclose(yl, yg[r["K0"]:r["K0"] + r["NK"]], rtol=1e-12, atol=1e-12 * np.abs(yg).max())
    its = {r["it"] for r in results}
    assert len(its) == 1 and all(r["conv"] for r in results), its
    it = its.pop()
    assert abs(it - ref["it"]) <= 1, (it, ref["it"])
