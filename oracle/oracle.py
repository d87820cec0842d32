"""ctypes front end of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` as
the checker, and by ``bench.py`` for the CPU-baseline leg.  The product path
never imports this module.

The functions restate the fem-rs reference algorithms; see femoracle.h for the
file:line each one follows.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

MASS, DIFF, MASS_DIFF = 1, 2, 3
ALL_FACES = 0x3F  # tags 1..6 (z0, z1, y0, y1, x0, x1)


class _Mesh(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("p", C.c_int),
                ("nq", C.c_int), ("vcoord", C.c_void_p)]


class _Cfg(C.Structure):
    _fields_ = [("precond", C.c_int), ("cheb_degree", C.c_int), ("lmin", C.c_double),
                ("lmax", C.c_double), ("rtol", C.c_double), ("atol", C.c_double),
                ("max_iter", C.c_int)]


class _Res(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int),
                ("final_residual", C.c_double), ("true_residual", C.c_double),
                ("applies", C.c_int64)]


def build() -> str:
    """Compile liboracle.so with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, i, d, i64 = C.c_void_p, C.c_int, C.c_double, C.c_int64
        L.or_ndofs.restype = i64
        L.or_ndofs.argtypes = [vp]
        L.or_pa_apply.argtypes = [vp, i, d, d, vp, d, vp, d, vp, vp, i, i]
        L.or_apply_constrained.argtypes = [vp, i, d, d, vp, d, vp, d, vp, vp, vp, i]
        L.or_element_matrix.argtypes = [vp, i64, i, d, d, vp, d, vp, d, vp]
        L.or_ess_mask.argtypes = [vp, i, vp]
        L.or_diagonal.argtypes = [vp, i, d, d, vp, d, vp, d, vp, vp, i]
        L.or_source.argtypes = [vp, i, i, vp, vp]
        L.or_l2_error_sin.restype = d
        L.or_l2_error_sin.argtypes = [vp, i, vp]
        L.or_lumped_mass.argtypes = [vp, vp, d, i, vp]
        L.or_tet_rule.argtypes = [i, vp, vp, i]
        L.or_tet_basis.argtypes = [i, vp, vp, vp]
        L.or_tet_pa_apply.argtypes = [i, i64, vp, i64, vp, i, d, d, vp, d, vp, d, i, vp, vp, vp, i]
        L.or_tet_diagonal.argtypes = [i, i64, vp, i64, vp, i, d, d, vp, d, vp, d, i, vp, vp]
        L.or_tet_source.argtypes = [i, i64, vp, i64, vp, i, vp, vp]
        L.or_tet_l2_error_sin.argtypes = [i, vp, i64, vp, i, vp]
        L.or_tet_l2_error_sin.restype = d
        L.or_lumped_mass.restype = i
        L.or_source.restype = i
        L.or_pcg.argtypes = [vp, i, d, d, vp, d, vp, d, vp, vp, vp, vp, vp, i]
        L.or_lambda_max.restype = d
        L.or_lambda_max.argtypes = [vp, i, d, d, vp, d, vp, d, vp, i, i]
        L.or_gauss_legendre.argtypes = [i, vp, vp]
        L.or_hex_rule_points.restype = i
        L.or_hex_rule_points.argtypes = [i]
        L.or_lagrange1d.argtypes = [i, d, vp, vp]
        L.or_hexq1_basis.argtypes = [vp, vp, vp]
        L.or_ref_chebyshev_smooth_csr.argtypes = [i64, vp, vp, vp, vp, vp, d, d, i]
        L.or_ref_spectral_radius_csr.restype = d
        L.or_ref_spectral_radius_csr.argtypes = [i64, vp, vp, vp, i]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


class Mesh:
    """Structured hex box: nx*ny*nz elements, order p, nq Gauss points per
    direction, optional vertex coordinates ((nx+1)(ny+1)(nz+1), 3)."""

    def __init__(self, nx, ny, nz, p, nq=None, vcoord=None):
        self.nx, self.ny, self.nz, self.p = int(nx), int(ny), int(nz), int(p)
        self.nq = int(nq if nq is not None else p + 1)
        self.vcoord = None if vcoord is None else np.ascontiguousarray(vcoord, dtype=np.float64)
        self._m = _Mesh(self.nx, self.ny, self.nz, self.p, self.nq, _p(self.vcoord))

    @property
    def ptr(self):
        return C.byref(self._m)

    @property
    def n_elem(self):
        return self.nx * self.ny * self.nz

    @property
    def shape(self):
        p = self.p
        return (self.nz * p + 1, self.ny * p + 1, self.nx * p + 1)

    @property
    def ndofs(self):
        return int(lib().or_ndofs(self.ptr))


class Coef:
    def __init__(self, kind=DIFF, c_m=1.0, c_k=1.0, kappa_q=None, kappa=1.0, rho_q=None, rho=1.0):
        self.kind, self.c_m, self.c_k = kind, float(c_m), float(c_k)
        self.kappa_q = None if kappa_q is None else np.ascontiguousarray(kappa_q, dtype=np.float64)
        self.rho_q = None if rho_q is None else np.ascontiguousarray(rho_q, dtype=np.float64)
        self.kappa, self.rho = float(kappa), float(rho)

    def args(self):
        return (self.kind, self.c_m, self.c_k, _p(self.kappa_q), self.kappa, _p(self.rho_q), self.rho)


def pa_apply(mesh, coef, x, y=None, accumulate=False, nthreads=0):
    x = np.ascontiguousarray(x, dtype=np.float64)
    if y is None:
        y = np.zeros(mesh.ndofs)
    rc = lib().or_pa_apply(mesh.ptr, *coef.args(), _p(x), _p(y), int(accumulate), nthreads)
    assert rc == 0, rc
    return y


def ess_mask(mesh, tag_bits=ALL_FACES):
    m = np.zeros(mesh.ndofs, dtype=np.uint8)
    lib().or_ess_mask(mesh.ptr, tag_bits, _p(m))
    return m


def apply_constrained(mesh, coef, ess, x, nthreads=0):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(mesh.ndofs)
    rc = lib().or_apply_constrained(mesh.ptr, *coef.args(), _p(ess), _p(x), _p(y), nthreads)
    assert rc == 0, rc
    return y


def diagonal(mesh, coef, ess=None, nthreads=0):
    d = np.zeros(mesh.ndofs)
    lib().or_diagonal(mesh.ptr, *coef.args(), _p(ess), _p(d), nthreads)
    return d


def element_matrix(mesh, e, coef):
    L = (mesh.p + 1) ** 3
    K = np.zeros((L, L))
    lib().or_element_matrix(mesh.ptr, int(e), *coef.args(), _p(K))
    return K


def source(mesh, ess=None, nq=None):
    b = np.zeros(mesh.ndofs)
    if lib().or_source(mesh.ptr, 1, int(nq if nq else mesh.p + 1), _p(ess), _p(b)) != 0:
        raise ValueError("the oracle's Gauss rules have 1 to 4 points")
    return b


def l2_error_sin(mesh, u, nq=None):
    """Default rule: p+2 points, clamped to 4 as hex_rule does (quadrature.rs:405-419)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    e = float(lib().or_l2_error_sin(mesh.ptr, int(nq if nq else min(mesh.p + 2, 4)), _p(u)))
    if e < 0:
        raise ValueError("the oracle's Gauss rules have 1 to 4 points")
    return e


def lumped_mass(mesh, rho_q=None, rho=1.0, nq=None):
    d = np.zeros(mesh.ndofs)
    rq = None if rho_q is None else np.ascontiguousarray(rho_q, dtype=np.float64)
    if lib().or_lumped_mass(mesh.ptr, _p(rq), C.c_double(rho), int(nq if nq else mesh.p + 1), _p(d)) != 0:
        raise ValueError("the oracle's Gauss rules have 1 to 4 points")
    return d


def lambda_max(mesh, coef, ess, iters=20, nthreads=0):
    return float(lib().or_lambda_max(mesh.ptr, *coef.args(), _p(ess), iters, nthreads))


def pcg(mesh, coef, ess, b, x0=None, precond=1, cheb_degree=4, lmin=0.0, lmax=0.0,
        rtol=1e-8, atol=0.0, max_iter=1000, nthreads=0):
    """Returns (x, dict(converged, iterations, final_residual, true_residual, applies))."""
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(mesh.ndofs) if x0 is None else np.array(x0, dtype=np.float64)
    cfg = _Cfg(precond, cheb_degree, lmin, lmax, rtol, atol, max_iter)
    res = _Res()
    lib().or_pcg(mesh.ptr, *coef.args(), _p(ess), _p(b), _p(x), C.byref(cfg), C.byref(res), nthreads)
    return x, dict(converged=bool(res.converged), iterations=res.iterations,
                   final_residual=res.final_residual, true_residual=res.true_residual,
                   applies=int(res.applies))


def assemble_csr(mesh, coef):
    """Assembled global matrix (scipy CSR) from oracle element matrices, as
    Assembler::assemble_bilinear does (crates/assembly/src/assembler.rs:409-429)."""
    import scipy.sparse as sp
    from itertools import product
    p, D = mesh.p, mesh.p + 1
    NZ, NJ, NI = mesh.shape
    L = D ** 3
    rows, cols, vals = [], [], []
    loc = np.array([(c * NJ + b) * NI + a for c, b, a in product(range(D), range(D), range(D))])
    for e in range(mesh.n_elem):
        ex, ey, ez = e % mesh.nx, (e // mesh.nx) % mesh.ny, e // (mesh.nx * mesh.ny)
        base = (ez * p * NJ + ey * p) * NI + ex * p
        g = base + loc
        K = element_matrix(mesh, e, coef)
        rows.append(np.repeat(g, L)); cols.append(np.tile(g, L)); vals.append(K.ravel())
    n = mesh.ndofs
    A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    return A.tocsr()


def gauss(n):
    x = np.zeros(n); w = np.zeros(n)
    lib().or_gauss_legendre(n, _p(x), _p(w))
    return x, w


def hex_rule_points(order):
    return int(lib().or_hex_rule_points(order))


def lagrange1d(p, xi):
    phi = np.zeros(p + 1); dphi = np.zeros(p + 1)
    lib().or_lagrange1d(p, float(xi), _p(phi), _p(dphi))
    return phi, dphi


def hexq1_basis(xi):
    xi = np.ascontiguousarray(xi, dtype=np.float64)
    phi = np.zeros(8); g = np.zeros(24)
    lib().or_hexq1_basis(_p(xi), _p(phi), _p(g))
    return phi, g.reshape(8, 3)


def ref_chebyshev_smooth_csr(A, x, b, lmin, lmax, n_iter):
    rp = np.ascontiguousarray(A.indptr, dtype=np.int64)
    ci = np.ascontiguousarray(A.indices, dtype=np.int64)
    v = np.ascontiguousarray(A.data, dtype=np.float64)
    x = np.array(x, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    lib().or_ref_chebyshev_smooth_csr(A.shape[0], _p(rp), _p(ci), _p(v), _p(x), _p(b), lmin, lmax, n_iter)
    return x


def ref_spectral_radius_csr(A, n_iter):
    rp = np.ascontiguousarray(A.indptr, dtype=np.int64)
    ci = np.ascontiguousarray(A.indices, dtype=np.int64)
    v = np.ascontiguousarray(A.data, dtype=np.float64)
    return float(lib().or_ref_spectral_radius_csr(A.shape[0], _p(rp), _p(ci), _p(v), n_iter))


# ---- tetrahedra (oracle/femoracle_tet.c) -------------------------------------
def tet_rule(order):
    pts = np.zeros((64, 3))
    w = np.zeros(64)
    n = lib().or_tet_rule(int(order), _p(pts), _p(w), 64)
    assert n > 0
    return pts[:n].copy(), w[:n].copy()


def tet_basis(p, xi):
    nl = {1: 4, 2: 10, 3: 20}[p]
    phi = np.zeros(nl)
    g = np.zeros((nl, 3))
    lib().or_tet_basis(int(p), _p(np.ascontiguousarray(xi, dtype=np.float64)), _p(phi), _p(g))
    return phi, g


class TetSpace:
    """An order-p tet space: coords [n_nodes, 3], elem_dofs [E, 4|10] (first 4 =
    vertex nodes), n_dofs, optional essential mask [n_dofs] uint8."""

    def __init__(self, p, coords, elem_dofs, n_dofs, ess=None):
        self.p = int(p)
        self.coords = np.ascontiguousarray(coords, dtype=np.float64)
        self.elem_dofs = np.ascontiguousarray(elem_dofs, dtype=np.int32)
        self.n_dofs = int(n_dofs)
        self.n_elem = self.elem_dofs.shape[0]
        self.ess = None if ess is None else np.ascontiguousarray(ess, dtype=np.uint8)


def _tet_coef(coef):
    kq = None if coef.kappa_q is None else np.ascontiguousarray(coef.kappa_q, dtype=np.float64)
    rq = None if coef.rho_q is None else np.ascontiguousarray(coef.rho_q, dtype=np.float64)
    return kq, rq


def tet_pa_apply(sp, coef, x, quad_order, constrained=False, y=None):
    kq, rq = _tet_coef(coef)
    x = np.ascontiguousarray(x, dtype=np.float64)
    acc = y is not None
    y = np.zeros(sp.n_dofs) if y is None else y
    rc = lib().or_tet_pa_apply(sp.p, sp.n_dofs, _p(sp.coords), sp.n_elem, _p(sp.elem_dofs), coef.kind,
                               coef.c_m, coef.c_k, _p(kq), coef.kappa, _p(rq), coef.rho, int(quad_order),
                               _p(sp.ess) if constrained else None, _p(x), _p(y), int(acc))
    assert rc == 0, rc
    return y


def tet_diagonal(sp, coef, quad_order, constrained=False):
    kq, rq = _tet_coef(coef)
    d = np.zeros(sp.n_dofs)
    rc = lib().or_tet_diagonal(sp.p, sp.n_dofs, _p(sp.coords), sp.n_elem, _p(sp.elem_dofs), coef.kind,
                               coef.c_m, coef.c_k, _p(kq), coef.kappa, _p(rq), coef.rho, int(quad_order),
                               _p(sp.ess) if constrained else None, _p(d))
    assert rc == 0, rc
    return d


def tet_source(sp, quad_order, constrained=True):
    b = np.zeros(sp.n_dofs)
    rc = lib().or_tet_source(sp.p, sp.n_dofs, _p(sp.coords), sp.n_elem, _p(sp.elem_dofs), int(quad_order),
                             _p(sp.ess) if constrained else None, _p(b))
    assert rc == 0, rc
    return b


def tet_l2_error_sin(sp, u, quad_order):
    u = np.ascontiguousarray(u, dtype=np.float64)
    return float(lib().or_tet_l2_error_sin(sp.p, _p(sp.coords), sp.n_elem, _p(sp.elem_dofs), int(quad_order),
                                            _p(u)))
