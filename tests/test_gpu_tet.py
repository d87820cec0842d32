"""Tetrahedral PA operator on the GPU (fg_tet_*) against the tetrahedral
oracle, the restatement of partial.rs's element loop on Tet4 with TetP1 /
TetP2 / TetP3: apply and diagonal <= 1e-12 relative (2-norm) on unit_cube_tet meshes
with perturbed interior nodes and per-point lognormal coefficients, all
operator kinds, accumulate / overwrite, constrained / raw, host and device
vectors; bit-for-bit repeatable; the 3-D Poisson known answers of
crates/assembly/tests/poisson.rs:495-533 reproduced with the GPU apply."""
import math

import numpy as np
import pytest

from conftest import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import femgpu  # noqa: E402
from femgpu import tet as T  # noqa: E402


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def space(n, p, perturb=0.25, seed=0):
    coords, dofs, nd, mask = T.unit_cube_space(n, p)
    if perturb:
        rng = np.random.default_rng(seed)
        inner = np.all((coords > 1e-12) & (coords < 1 - 1e-12), axis=1)
        coords = coords.copy()
        coords[inner] += perturb / n * rng.uniform(-1, 1, size=(inner.sum(), 3))
    return coords, dofs, nd, mask


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("kind", [femgpu.MASS, femgpu.DIFF, femgpu.MASS_DIFF])
def test_tet_apply_matches_oracle(p, kind):
    need_gpu()
    coords, dofs, nd, mask = space(5 if p < 3 else 3, p, seed=p + kind)
    qo = 2 * p + (1 if kind & 1 else 0)
    nq = len(O.tet_rule(qo)[1])
    rng = np.random.default_rng(kind)
    kq = np.exp(rng.normal(size=dofs.shape[0] * nq))
    rq = np.exp(0.3 * rng.normal(size=dofs.shape[0] * nq))
    op = femgpu.TetOperator(p, coords, dofs, nd, kind=kind, kappa=kq, rho=rq, c_mass=0.7, c_diff=1.3,
                            quad_order=qo, ess=mask)
    assert op.nq == nq and op.n_dofs() == nd
    sp = O.TetSpace(p, coords, dofs, nd, mask)
    coef = O.Coef(kind, c_m=0.7, c_k=1.3, kappa_q=kq, rho_q=rq)
    x = rng.standard_normal(nd)
    for constrained in (False, True):
        ref = O.tet_pa_apply(sp, coef, x, qo, constrained)
        y = op.matvec(x, constrained)
        assert rel(y, ref) <= 1e-12, (constrained, rel(y, ref))
        y2 = np.ones(nd)
        op.apply(x, y2, constrained)
        assert rel(y2, ref + 1.0) <= 1e-12
        assert rel(op.diagonal(constrained), O.tet_diagonal(sp, coef, qo, constrained)) <= 1e-12
    assert np.array_equal(op.matvec(x), op.matvec(x))
    # device vectors
    xd = torch.tensor(x, device="cuda")
    yd = torch.zeros_like(xd)
    op.apply_zero(xd, yd, True)
    assert rel(yd.cpu().numpy(), O.tet_pa_apply(sp, coef, x, qo, True)) <= 1e-12


@pytest.mark.parametrize("p", [1, 2, 3])
def test_tet_single_cube_and_single_element(p):
    """Smallest meshes: the 6 tets of one cube, and one tetrahedron alone."""
    need_gpu()
    coords, dofs, nd, mask = space(1, p, perturb=0.0)
    sp = O.TetSpace(p, coords, dofs, nd, mask)
    op = femgpu.TetOperator(p, coords, dofs, nd, kind=femgpu.MASS_DIFF, quad_order=2 * p, ess=mask)
    x = np.random.default_rng(p).standard_normal(nd)
    coef = O.Coef(femgpu.MASS_DIFF)
    for constrained in (False, True):
        assert rel(op.matvec(x, constrained), O.tet_pa_apply(sp, coef, x, 2 * p, constrained)) <= 1e-12
    one = dofs[:1]
    used = np.unique(one)
    remap = np.full(nd, -1)
    remap[used] = np.arange(len(used))
    c1 = coords[used[used < len(coords)]] if p == 1 else None
    if p == 1:
        d1 = remap[one].astype(np.int32)
        op1 = femgpu.TetOperator(1, c1, d1, 4)
        sp1 = O.TetSpace(1, c1, d1, 4)
        x1 = np.arange(1.0, 5.0)
        assert rel(op1.matvec(x1), O.tet_pa_apply(sp1, O.Coef(O.DIFF), x1, 2)) <= 1e-12


def test_tet_quadrature_points():
    need_gpu()
    coords, dofs, nd, mask = space(3, 2, seed=9)
    op = femgpu.TetOperator(2, coords, dofs, nd, quad_order=5)
    pts, _ = O.tet_rule(5)
    xyz = op.quadrature_points()
    x0 = coords[dofs[:, 0]]
    J = np.stack([coords[dofs[:, c + 1]] - x0 for c in range(3)], axis=2)  # [E, 3(row), 3(col)]
    ref = x0[:, None, :] + np.einsum("erc,qc->eqr", J, pts)
    assert np.abs(xyz - ref).max() < 1e-14


def _gpu_poisson_l2(n, p):
    coords, dofs, nd, mask = space(n, p, perturb=0.0)
    qo = 2 * p + 1
    op = femgpu.TetOperator(p, coords, dofs, nd, quad_order=qo, ess=mask)
    sp = O.TetSpace(p, coords, dofs, nd, mask)
    b = O.tet_source(sp, qo)
    # CG driven from the host, every operator application on the GPU
    x = np.zeros(nd)
    r = b.copy()
    pv = r.copy()
    rr = r @ r
    for _ in range(5000):
        ap = op.matvec(pv, True)
        a = rr / (pv @ ap)
        x += a * pv
        r -= a * ap
        rn = r @ r
        if math.sqrt(rn) < 1e-12 * math.sqrt(b @ b):
            break
        pv = r + (rn / rr) * pv
        rr = rn
    return O.tet_l2_error_sin(sp, x, 2 * p + 2)


def test_tet_poisson_known_answers_with_gpu_apply():
    need_gpu()
    e4, e8 = _gpu_poisson_l2(4, 1), _gpu_poisson_l2(8, 1)
    assert e4 < 1e-1 and math.log2(e4 / e8) > 1.8
    assert _gpu_poisson_l2(4, 2) < 1e-2
    assert _gpu_poisson_l2(4, 3) < 5e-3


def test_tet_rejects_bad_input():
    need_gpu()
    coords, dofs, nd, mask = space(2, 1, perturb=0.0)
    bad = dofs.copy()
    bad[0, 0] = nd + 5
    with pytest.raises(femgpu.SolverError):
        femgpu.TetOperator(1, coords, bad, nd)
    with pytest.raises(femgpu.SolverError):
        femgpu.TetOperator(4, coords, dofs, nd)
    op = femgpu.TetOperator(1, coords, dofs, nd)
    with pytest.raises(femgpu.SolverError):
        op.matvec(np.ones(nd), constrained=True)  # no essential mask given


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("kind", [femgpu.DIFF, femgpu.MASS_DIFF])
@pytest.mark.parametrize("chunk", [32, 96, None])
def test_tet_chunk_plans_on_shuffled_mesh(p, kind, chunk, monkeypatch):
    """The chunked scatter with many chunks (most DOFs shared between chunks):
    elements given in a random order, DOFs renumbered at random, two DOFs that
    no element touches, an arbitrary essential list; apply, accumulate and
    diagonal against the oracle, and bit-for-bit repeatable."""
    need_gpu()
    if chunk:
        monkeypatch.setenv("FG_TET_CHUNK", str(chunk))
    else:
        monkeypatch.delenv("FG_TET_CHUNK", raising=False)
    coords, dofs, nd, _ = space(6 if p < 3 else 4, p, seed=11 + p)
    rng = np.random.default_rng(100 * p + kind)
    n_nodes = coords.shape[0]
    # vertex DOFs must stay the nodes 0..n_nodes-1: permute the nodes and the other DOFs separately
    pn = rng.permutation(n_nodes)
    po = n_nodes + rng.permutation(nd - n_nodes)
    newid = np.concatenate([pn, po])
    coords2 = np.empty_like(coords)
    coords2[pn] = coords
    dofs2 = newid[dofs][rng.permutation(dofs.shape[0])].astype(np.int32)
    nd2 = nd + 2
    mask = np.zeros(nd2, dtype=np.uint8)
    mask[rng.choice(nd, size=nd // 7, replace=False)] = 1
    mask[nd] = 1  # an untouched essential DOF
    qo = 2 * p
    nq = len(O.tet_rule(qo)[1])
    kq = np.exp(rng.normal(size=dofs2.shape[0] * nq))
    op = femgpu.TetOperator(p, coords2, dofs2, nd2, kind=kind, kappa=kq, c_mass=0.9, c_diff=1.1,
                            quad_order=qo, ess=mask)
    sp = O.TetSpace(p, coords2, dofs2, nd2, mask)
    coef = O.Coef(kind, c_m=0.9, c_k=1.1, kappa_q=kq)
    x = rng.standard_normal(nd2)
    for constrained in (False, True):
        ref = O.tet_pa_apply(sp, coef, x, qo, constrained)
        y = op.matvec(x, constrained)
        assert rel(y, ref) <= 1e-12, (constrained, rel(y, ref))
        y2 = np.full(nd2, 0.5)
        op.apply(x, y2, constrained)
        assert rel(y2, ref + 0.5) <= 1e-12
        assert rel(op.diagonal(constrained), O.tet_diagonal(sp, coef, qo, constrained)) <= 1e-12
    assert np.array_equal(op.matvec(x, True), op.matvec(x, True))
