"""Golden vectors of the PA operator path (tests/golden/hex_pa_golden.npz,
written by tests/golden/make_golden.py from the oracle).

CPU: the oracle reproduces the stored vectors (guards the checker itself
against drift).  GPU: the sm_100a library, through the C ABI, matches them --
FP64 apply and diagonal to 1e-12 relative (2-norm), Jacobi-PCG iteration
counts within +-1 and the solution to 1e-8.
"""
import os
import sys

import numpy as np
import pytest

from conftest import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as G  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "hex_pa_golden.npz"))
CASES = list(G.cases())
IDS = [G.case_key(*c) for c in CASES]


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def stored(key):
    pre = key + "/"
    return {k[len(pre):]: GOLD[k] for k in GOLD.files if k.startswith(pre)}


@pytest.mark.parametrize("p,shape,name", CASES, ids=IDS)
def test_oracle_reproduces_golden(p, shape, name):
    g = stored(G.case_key(p, shape, name))
    out = G.oracle_case(p, shape, name, g["vc"], g["kq"], g["rq"], g["x"])
    for k in ("y", "yc", "d", "b", "xs"):
        if k in out:
            assert relerr(out[k], g[k]) <= 1e-14, (k, relerr(out[k], g[k]))
    if "it" in out:
        assert int(out["it"]) == int(g["it"])


@pytest.mark.gpu
@pytest.mark.parametrize("p,shape,name", CASES, ids=IDS)
def test_gpu_matches_golden(p, shape, name):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import femgpu

    g = stored(G.case_key(p, shape, name))
    nx, ny, nz = shape
    kind = {"mass": femgpu.MASS, "diff": femgpu.DIFF, "massdiff": femgpu.MASS_DIFF}[name]
    op = femgpu.PAOperator(dict(nx=nx, ny=ny, nz=nz, vcoord=g["vc"]), p, kind, kappa=g["kq"], rho=g["rq"],
                           c_mass=G.C_M, c_diff=G.C_K, ess_tags=femgpu.TAG_ALL)
    try:
        assert relerr(op.matvec(g["x"]), g["y"]) <= 1e-12
        assert relerr(op.matvec(g["x"], constrained=True), g["yc"]) <= 1e-12
        assert relerr(op.diagonal(constrained=True), g["d"]) <= 1e-12
        if "it" in g:
            xs = np.zeros(op.n_dofs())
            res = femgpu.solve_pcg_jacobi(op, g["b"], xs, femgpu.SolverConfig(rtol=1e-10, max_iter=5000))
            assert res.converged
            assert abs(res.iterations - int(g["it"])) <= 1, (res.iterations, int(g["it"]))
            assert relerr(xs, g["xs"]) <= 1e-8
    finally:
        op.close()
