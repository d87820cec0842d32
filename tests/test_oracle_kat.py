"""Pins the CPU oracle against the fem-rs reference's own known-answer tests.

The reference ships no golden vectors for the PA path, so each test below
restates one of its unit/integration tests (file:line cited) on the hex
elements this project builds.  CPU only.
"""
import math

import numpy as np
import pytest

from conftest import oracle as O


def perturbed_vertices(nx, ny, nz, amp=0.15, seed=0):
    """Unit-cube vertex grid with interior vertices jittered (non-affine hexes)."""
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    v = np.stack([i / nx, j / ny, k / nz], axis=-1).astype(np.float64)
    h = np.array([1 / nx, 1 / ny, 1 / nz])
    interior = (i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)
    v[interior] += amp * h * rng.uniform(-1, 1, size=(interior.sum(), 3))
    return v.reshape(-1, 3)


# --- crates/element/src/quadrature.rs:421+ (weight sums) -------------------
@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_gauss_weights_and_hex_rule(n):
    x, w = O.gauss(n)
    assert abs(w.sum() - 2.0) < 1e-14
    # exact for degree 2n-1
    for deg in range(2 * n):
        exact = 0.0 if deg % 2 else 2.0 / (deg + 1)
        assert abs((w * x ** deg).sum() - exact) < 1e-14
    assert abs(w.sum() ** 3 - 8.0) < 1e-13  # hex weights sum to 8


def test_hex_rule_point_count():
    # quadrature.rs:405-419: n = clamp((order+2)/2, 1, 4); order 2p+1 -> p+1
    for p in (1, 2, 3):
        assert O.hex_rule_points(2 * p + 1) == p + 1
    assert O.hex_rule_points(0) == 1 and O.hex_rule_points(9) == 4


# --- crates/element/src/lagrange/hex.rs:72-113 -----------------------------
def test_hexq1_pou_grad_kronecker():
    x, _ = O.gauss(3)
    for xi in [(a, b, c) for a in x for b in x for c in x]:
        phi, g = O.hexq1_basis(xi)
        assert abs(phi.sum() - 1.0) < 1e-12
        assert np.abs(g.sum(axis=0)).max() < 1e-11
    nodes = [(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1),
             (-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)]
    for i, nd in enumerate(nodes):
        phi, _ = O.hexq1_basis(nd)
        assert np.abs(phi - np.eye(8)[i]).max() < 1e-13


def test_lagrange1d_matches_reference_formulas():
    for xv in np.linspace(-1, 1, 7):
        # quad.rs:92-105
        phi, dphi = O.lagrange1d(2, xv)
        assert np.allclose(phi, [0.5 * xv * (xv - 1), 1 - xv * xv, 0.5 * xv * (xv + 1)], atol=1e-15)
        assert np.allclose(dphi, [0.5 * (2 * xv - 1), -2 * xv, 0.5 * (2 * xv + 1)], atol=1e-15)
        # hex.rs Q1 factors (1 -+ x)/2
        phi, dphi = O.lagrange1d(1, xv)
        assert np.allclose(phi, [(1 - xv) / 2, (1 + xv) / 2], atol=1e-15)
        # seg.rs:100-121 SegP3 on [0,1] with nodes 0, 1, 1/3, 2/3 (mapped t = (x+1)/2)
        t = (xv + 1) / 2
        ref = [-4.5 * t ** 3 + 9 * t * t - 5.5 * t + 1, 4.5 * t ** 3 - 4.5 * t * t + t,
               13.5 * t ** 3 - 22.5 * t * t + 9 * t, -13.5 * t ** 3 + 18 * t * t - 4.5 * t]
        phi, _ = O.lagrange1d(3, xv)
        assert np.allclose(phi, [ref[0], ref[2], ref[3], ref[1]], atol=1e-14)
        # partition of unity, derivative sum zero
        for p in (1, 2, 3):
            phi, dphi = O.lagrange1d(p, xv)
            assert abs(phi.sum() - 1) < 1e-14 and abs(dphi.sum()) < 1e-13


# --- crates/assembly/src/partial.rs:322-366 (PA vs assembled, <= 1e-11) -----
@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("kind", [O.MASS, O.DIFF, O.MASS_DIFF])
def test_pa_matches_assembled(p, kind):
    n = 3
    m = O.Mesh(n, n, 2, p, vcoord=perturbed_vertices(n, n, 2, seed=p))
    rng = np.random.default_rng(10 + p)
    kq = np.exp(rng.normal(size=m.n_elem * m.nq ** 3))
    coef = O.Coef(kind, c_m=1.3, c_k=0.7, kappa_q=kq, rho=2.0)
    A = O.assemble_csr(m, coef)
    for x in (np.ones(m.ndofs), rng.normal(size=m.ndofs)):
        y = O.pa_apply(m, coef, x)
        ya = A @ x
        assert np.linalg.norm(y - ya) < 1e-11 * max(1.0, np.linalg.norm(ya))


# --- partial.rs:380-392 (K 1 = 0), standard/diffusion.rs:57-118 ------------
@pytest.mark.parametrize("p", [1, 2, 3])
def test_diffusion_constant_nullspace_and_symmetry(p):
    m = O.Mesh(3, 2, 2, p, vcoord=perturbed_vertices(3, 2, 2, seed=3))
    coef = O.Coef(O.DIFF, kappa=1.0)
    y = O.pa_apply(m, coef, np.ones(m.ndofs))
    assert np.abs(y).max() < 1e-12
    K = O.element_matrix(m, 5, coef)
    assert np.abs(K - K.T).max() < 1e-12
    assert np.abs(K.sum(axis=1)).max() < 1e-12


# --- partial.rs:394-412 (linearity, <= 1e-13) -------------------------------
def test_pa_linearity():
    m = O.Mesh(3, 3, 3, 2)
    coef = O.Coef(O.MASS)
    n = m.ndofs
    x = np.arange(n) / n
    y1 = O.pa_apply(m, coef, x)
    y2 = O.pa_apply(m, coef, x)
    ysum = O.pa_apply(m, coef, x, y=y1.copy(), accumulate=True)
    assert np.linalg.norm(ysum - 2 * y2) < 1e-13
    assert np.linalg.norm(y1 - y2) == 0.0  # deterministic scatter


# --- standard/mass.rs:67-82 (1'M1 = |Omega|, <= 1e-10) ----------------------
@pytest.mark.parametrize("p", [1, 2, 3])
def test_mass_total(p):
    m = O.Mesh(2, 3, 2, p, vcoord=perturbed_vertices(2, 3, 2, seed=7))
    one = np.ones(m.ndofs)
    assert abs(one @ O.pa_apply(m, O.Coef(O.MASS), one) - 1.0) < 1e-10


def test_thread_count_independence():
    m = O.Mesh(6, 5, 4, 2)
    coef = O.Coef(O.DIFF)
    x = np.random.default_rng(1).normal(size=m.ndofs)
    assert np.array_equal(O.pa_apply(m, coef, x, nthreads=1), O.pa_apply(m, coef, x, nthreads=4))


# --- examples/mfem_ex1_poisson.rs:184-237 on hexes --------------------------
def _solve_ex1(n, p, scale=1.0, rtol=1e-10):
    m = O.Mesh(n, n, n, p)
    ess = O.ess_mask(m)
    b = scale * O.source(m, ess)
    coef = O.Coef(O.DIFF)
    x, info = O.pcg(m, coef, ess, b, precond=1, rtol=rtol, max_iter=5000)
    return m, x, info


def test_ex1_coarse_error_and_rate():
    m8, x8, i8 = _solve_ex1(8, 1)
    m16, x16, i16 = _solve_ex1(16, 1)
    assert i8["converged"] and i16["converged"]
    assert i8["final_residual"] < 1e-8
    e8, e16 = O.l2_error_sin(m8, x8), O.l2_error_sin(m16, x16)
    assert e8 < 2.2e-2
    assert math.log(e8 / e16) / math.log(2.0) > 1.5
    _, x82, _ = _solve_ex1(8, 2)
    assert O.l2_error_sin(O.Mesh(8, 8, 8, 2), x82) < e8


def test_ex1_sign_symmetry():
    m, xp, _ = _solve_ex1(6, 1, 1.0)
    _, xn, _ = _solve_ex1(6, 1, -1.0)
    assert abs(np.linalg.norm(xp) - np.linalg.norm(xn)) / np.linalg.norm(xp) < 1e-12
    assert abs(O.l2_error_sin(m, xp) - O.l2_error_sin(m, -xn)) < 1e-12


def test_pcg_matches_dense_solve():
    m = O.Mesh(4, 3, 3, 2)
    ess = O.ess_mask(m)
    coef = O.Coef(O.DIFF, kappa_q=np.exp(np.random.default_rng(2).normal(size=m.n_elem * 27)))
    b = O.source(m, ess)
    x, info = O.pcg(m, coef, ess, b, precond=1, rtol=1e-13, max_iter=2000)
    A = O.assemble_csr(m, coef).toarray()
    free = ess == 0
    xd = np.zeros(m.ndofs)
    xd[free] = np.linalg.solve(A[np.ix_(free, free)], b[free])
    assert info["converged"]
    assert np.abs(x - xd).max() < 1e-10 * np.abs(xd).max()


def _cg_operator_numpy(A, b, x, rtol, atol, max_iter):
    """crates/solver/src/lib.rs:198-278 restated on an assembled matrix:
    (converged, iterations, final_residual) with the absolute residual."""
    r = b - A @ x
    p = r.copy()
    tol = max(atol, rtol * max(np.linalg.norm(b), 1e-32))
    rs_old = r @ r
    res = np.sqrt(rs_old)
    if res <= tol:
        return True, 0, res
    for it in range(max_iter):
        ap = A @ p
        pap = p @ ap
        if abs(pap) < 1e-32:
            return False, it, res
        alpha = rs_old / pap
        x += alpha * p
        r -= alpha * ap
        rs_new = r @ r
        res = np.sqrt(rs_new)
        if res <= tol:
            return True, it + 1, res
        p = r + (rs_new / rs_old) * p
        rs_old = rs_new
    return False, max_iter, res


def _constrained_csr(m, coef, ess):
    A = O.assemble_csr(m, coef).tolil()
    fixed = np.nonzero(ess)[0]
    A[fixed, :] = 0.0
    A[:, fixed] = 0.0
    A[fixed, fixed] = 1.0
    return A.tocsr()


@pytest.mark.parametrize("rtol,atol", [(1e-9, 0.0), (1e-3, 0.0), (1e-12, 1e-4)])
def test_operator_cg_stopping_rule(rtol, atol):
    """precond 0 follows solve_cg_operator: tol = max(atol, rtol*max(||b||,
    1e-32)), ||r|| <= tol, absolute final residual."""
    m = O.Mesh(5, 4, 3, 2)
    ess = O.ess_mask(m)
    coef = O.Coef(O.DIFF, kappa_q=np.exp(np.random.default_rng(7).normal(size=m.n_elem * 27)))
    b = O.source(m, ess)
    x, info = O.pcg(m, coef, ess, b, precond=0, rtol=rtol, atol=atol, max_iter=2000)
    conv, its, res = _cg_operator_numpy(_constrained_csr(m, coef, ess), b, np.zeros(m.ndofs), rtol, atol, 2000)
    assert info["converged"] and conv
    assert abs(info["iterations"] - its) <= 1
    tol = max(atol, rtol * np.linalg.norm(b))
    # absolute residuals at the stop, both under the same tolerance
    assert info["final_residual"] <= tol and res <= tol
    assert info["final_residual"] > 0.05 * tol


def test_operator_cg_exits_before_first_iteration():
    m = O.Mesh(4, 4, 4, 1)
    ess = O.ess_mask(m)
    coef = O.Coef(O.DIFF)
    b = O.source(m, ess)
    x, _ = O.pcg(m, coef, ess, b, precond=1, rtol=1e-14, max_iter=2000)
    _, info = O.pcg(m, coef, ess, b, x0=x, precond=0, rtol=1e-6)
    assert info["converged"] and info["iterations"] == 0


def test_chebyshev_pcg_converges_faster():
    m = O.Mesh(8, 8, 8, 2)
    ess = O.ess_mask(m)
    coef = O.Coef(O.DIFF, kappa_q=np.exp(np.random.default_rng(4).normal(size=m.n_elem * 27)))
    b = O.source(m, ess)
    _, ij = O.pcg(m, coef, ess, b, precond=1, rtol=1e-8)
    lmax = 1.1 * O.lambda_max(m, coef, ess, iters=20)
    x, ic = O.pcg(m, coef, ess, b, precond=2, cheb_degree=4, lmin=lmax / 30, lmax=lmax, rtol=1e-8)
    assert ic["converged"] and ij["converged"]
    assert ic["iterations"] < ij["iterations"]
    assert ic["true_residual"] < 1e-8 * 1.01


# --- crates/amg/src/lib.rs:254-286 (reference Chebyshev compat) -------------
def _laplacian_1d(n):
    import scipy.sparse as sp
    return sp.diags([-np.ones(n - 1), 2 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1]).tocsr()


def test_ref_spectral_radius_estimate():
    rho = O.ref_spectral_radius_csr(_laplacian_1d(50), 30)
    assert 3.5 < rho < 4.1


def test_ref_chebyshev_reduces_residual():
    A = _laplacian_1d(50)
    b = np.ones(50)
    rho = O.ref_spectral_radius_csr(A, 20)
    lmax = rho * 1.1
    x = O.ref_chebyshev_smooth_csr(A, np.zeros(50), b, lmax / 30, lmax, 20)
    assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 0.9
