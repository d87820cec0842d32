"""The tetrahedral oracle pinned by the reference's own known-answer tests:
tet_rule weight sums (crates/element/src/quadrature.rs:451-456, 565-572),
TetP1/TetP2 partition of unity, zero gradient sum and Kronecker property at
the DOF points (crates/element/src/lagrange/tet.rs:451-497), the PA
properties of partial.rs:322-412 (symmetry, K 1 = 0, linearity, 1^T M 1 =
|Omega|), and the 3-D Poisson known answers of crates/assembly/tests/
poisson.rs:495-533 on unit_cube_tet (TetP1 L2 < 1e-1 at n = 4, rate > 1.8;
TetP2 L2 < 1e-2 and TetP3 L2 < 5e-3 at n = 4), solved here through the
oracle's PA apply.
The mesh and the P2 DOF map come from femgpu.tet (simplex.rs:591-679,
dof_manager.rs:628-700)."""
import math

import numpy as np
import pytest

from conftest import oracle as O
from femgpu import tet as T


@pytest.mark.parametrize("order", [1, 2, 3, 5, 6, 7])
def test_tet_rule_weight_sums(order):
    pts, w = O.tet_rule(order)
    assert abs(w.sum() - 1.0 / 6.0) < 1e-12
    assert np.all(pts >= 0) and np.all(pts.sum(axis=1) <= 1 + 1e-15)


@pytest.mark.parametrize("order,deg", [(1, 1), (2, 2), (5, 5), (7, 7)])
def test_tet_rule_exactness(order, deg):
    # integral of x^a y^b z^c over the unit tet = a! b! c! / (a+b+c+3)!
    pts, w = O.tet_rule(order)
    for a in range(deg + 1):
        for b in range(deg + 1 - a):
            c = deg - a - b
            exact = math.factorial(a) * math.factorial(b) * math.factorial(c) / math.factorial(a + b + c + 3)
            got = np.sum(w * pts[:, 0] ** a * pts[:, 1] ** b * pts[:, 2] ** c)
            assert abs(got - exact) < 1e-13


def _ref_nodes(p):
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)
    if p == 1:
        return v
    ed = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    if p == 2:
        return np.vstack([v] + [0.5 * (v[a] + v[b]) for a, b in ed])
    out = [v]
    for a, b in ed:
        out += [(2 * v[a] + v[b]) / 3, (v[a] + 2 * v[b]) / 3]
    out += [v[list(f)].mean(axis=0) for f in ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3))]
    return np.vstack(out)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_tet_basis_pou_grad_kronecker(p):
    nodes = _ref_nodes(p)
    pts, _ = O.tet_rule(7)
    for xi in pts:
        phi, g = O.tet_basis(p, xi)
        assert abs(phi.sum() - 1) < 1e-13 and np.abs(g.sum(axis=0)).max() < 1e-13
    for i, xi in enumerate(nodes):
        phi, _ = O.tet_basis(p, xi)
        assert np.abs(phi - np.eye(len(nodes))[i]).max() < 1e-14


def _space(n, p, perturb=0.0, seed=0):
    coords, dofs, nd, mask = T.unit_cube_space(n, p)
    if perturb:
        rng = np.random.default_rng(seed)
        inner = np.all((coords > 1e-12) & (coords < 1 - 1e-12), axis=1)
        coords = coords.copy()
        coords[inner] += perturb / n * rng.uniform(-1, 1, size=(inner.sum(), 3))
    return O.TetSpace(p, coords, dofs, nd, mask)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_tet_pa_properties(p):
    sp = _space(3, p, perturb=0.2, seed=p)
    nq = sum(1 for _ in range(len(O.tet_rule(2 * p)[1])))
    kq = np.exp(np.random.default_rng(1).normal(size=sp.n_elem * nq))
    K = O.Coef(O.DIFF, kappa_q=kq)
    ones = np.ones(sp.n_dofs)
    assert np.abs(O.tet_pa_apply(sp, K, ones, 2 * p)).max() < 1e-12
    rng = np.random.default_rng(2)
    x, z = rng.standard_normal(sp.n_dofs), rng.standard_normal(sp.n_dofs)
    kx, kz = O.tet_pa_apply(sp, K, x, 2 * p), O.tet_pa_apply(sp, K, z, 2 * p)
    assert abs(z @ kx - x @ kz) < 1e-12 * abs(z @ kx)
    lin = O.tet_pa_apply(sp, K, 2 * x - 3 * z, 2 * p)
    assert np.abs(lin - (2 * kx - 3 * kz)).max() < 1e-13 * np.abs(kx).max() * 10
    M = O.Coef(O.MASS)
    assert abs(ones @ O.tet_pa_apply(sp, M, ones, 2 * p) - 1.0) < 1e-12
    # diagonal = e_i^T A e_i
    d = O.tet_diagonal(sp, K, 2 * p)
    for i in rng.choice(sp.n_dofs, 5, replace=False):
        e = np.zeros(sp.n_dofs)
        e[i] = 1
        assert abs(O.tet_pa_apply(sp, K, e, 2 * p)[i] - d[i]) < 1e-13 * abs(d[i])


def _solve_poisson(n, p):
    from scipy.sparse.linalg import LinearOperator, cg
    sp = _space(n, p)
    qo = 2 * p + 1  # tests/poisson.rs:505
    b = O.tet_source(sp, qo)
    A = LinearOperator((sp.n_dofs,) * 2, matvec=lambda v: O.tet_pa_apply(sp, O.Coef(O.DIFF), v, qo, True))
    x, info = cg(A, b, rtol=1e-12, atol=0.0, maxiter=5000)
    assert info == 0
    return O.tet_l2_error_sin(sp, x, 2 * p + 2)


def test_poisson_tet_known_answers():
    e4 = _solve_poisson(4, 1)
    e8 = _solve_poisson(8, 1)
    assert e4 < 1e-1 and math.log2(e4 / e8) > 1.8
    assert _solve_poisson(4, 2) < 1e-2
    assert _solve_poisson(4, 3) < 5e-3  # tests/poisson.rs:536-541


def test_p3_dof_map_matches_build_p3_tet():
    """p3_dofs against a literal restatement of build_p3_tet's two passes."""
    c, conn = T.unit_cube_tet(2)
    d, nd = T.p3_dofs(conn, len(c))
    nn = len(c)
    em, fm, nxt, ref = {}, {}, nn, []
    for e in conn:
        n0, n1, n2, n3 = (int(v) for v in e)
        row = [n0, n1, n2, n3]
        for a, b in ((n0, n1), (n0, n2), (n0, n3), (n1, n2), (n1, n3), (n2, n3)):
            k = (min(a, b), max(a, b))
            if k not in em:
                em[k] = [nxt, nxt + 1]
                nxt += 2
            row += em[k] if a == k[0] else em[k][::-1]
        ref.append(row)
    for i, e in enumerate(conn):
        n0, n1, n2, n3 = (int(v) for v in e)
        for f in ((n0, n1, n2), (n0, n1, n3), (n0, n2, n3), (n1, n2, n3)):
            k = tuple(sorted(f))
            if k not in fm:
                fm[k] = nxt
                nxt += 1
            ref[i].append(fm[k])
    assert np.array_equal(np.array(ref), d) and nxt == nd
