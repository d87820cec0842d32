"""Writes tests/golden/hex_pa_golden.npz: golden input/output vectors of the
partial-assembly operator path, computed by the CPU oracle (the C restatement
of crates/assembly/src/partial.rs with the Hex8 geometry of
crates/assembly/src/assembler.rs:96-143, pinned by the reference's own
known-answer tests in tests/test_oracle_kat.py).

Cases: orders 1-3 on a perturbed 3x2x2 hex box (a second, 5x4x3 box for the
solver), mass, diffusion and mass + diffusion, per-quadrature-point kappa and
rho.  Stored per case: the inputs (vertex coordinates, coefficient tables, x)
and the oracle's unconstrained apply, constrained apply (all six faces
essential), constrained diagonal, load vector of the manufactured source,
and Jacobi-PCG (rtol 1e-10) solution and iteration count.

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402

KINDS = {"mass": O.MASS, "diff": O.DIFF, "massdiff": O.MASS_DIFF}
C_M, C_K = 1.7, 0.9


def perturbed_vertices(nx, ny, nz, seed, amp=0.15):
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    v = np.stack([i / nx, j / ny, k / nz], axis=-1).astype(np.float64)
    h = np.array([1 / nx, 1 / ny, 1 / nz])
    inner = (i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)
    v[inner] += amp * h * rng.uniform(-1, 1, size=(inner.sum(), 3))
    return v.reshape(-1, 3)


def cases():
    for p in (1, 2, 3):
        for shape in ((3, 2, 2), (5, 4, 3)):
            for name in KINDS:
                if shape == (5, 4, 3) and name != "diff":
                    continue
                yield p, shape, name


def case_key(p, shape, name):
    return f"p{p}_{shape[0]}x{shape[1]}x{shape[2]}_{name}"


def oracle_case(p, shape, name, vc, kq, rq, x):
    nx, ny, nz = shape
    mesh = O.Mesh(nx, ny, nz, p, vcoord=vc)
    coef = O.Coef(KINDS[name], c_m=C_M, c_k=C_K, kappa_q=kq, kappa=1.0, rho_q=rq, rho=1.0)
    ess = O.ess_mask(mesh)
    out = dict(y=O.pa_apply(mesh, coef, x), yc=O.apply_constrained(mesh, coef, ess, x),
               d=O.diagonal(mesh, coef, ess))
    if name == "diff":
        b = O.source(mesh, ess)
        xs, info = O.pcg(mesh, coef, ess, b, precond=1, rtol=1e-10, max_iter=5000)
        out.update(b=b, xs=xs, it=np.array(info["iterations"]))
    return out


def inputs(p, shape, name):
    nx, ny, nz = shape
    seed = 10 * p + sum(shape) + len(name)
    rng = np.random.default_rng(seed)
    E, q3 = nx * ny * nz, (p + 1) ** 3
    vc = perturbed_vertices(nx, ny, nz, seed)
    kq = np.exp(rng.normal(size=E * q3))
    rq = np.exp(0.3 * rng.normal(size=E * q3))
    ndofs = (nx * p + 1) * (ny * p + 1) * (nz * p + 1)
    x = rng.normal(size=ndofs)
    return vc, kq, rq, x


def main():
    data = {}
    for p, shape, name in cases():
        key = case_key(p, shape, name)
        vc, kq, rq, x = inputs(p, shape, name)
        data.update({f"{key}/vc": vc, f"{key}/kq": kq, f"{key}/rq": rq, f"{key}/x": x})
        for k, v in oracle_case(p, shape, name, vc, kq, rq, x).items():
            data[f"{key}/{k}"] = v
    path = os.path.join(HERE, "hex_pa_golden.npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path}: {len(data)} arrays")


if __name__ == "__main__":
    main()
