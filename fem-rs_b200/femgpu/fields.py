"""Synthetic inputs of the benchmark configurations.

``lognormal_kappa_q``: kappa(x) = exp(g(x)) at the quadrature points, where g is
a zero-mean Gaussian random field with variance sigma2 and squared-exponential
correlation exp(-|d|^2 / (2 ell^2)).  The SE kernel is separable, so on the
tensor grid of quadrature-point coordinates g = sigma (Lz (x) Ly (x) Lx) xi
with L L^T the 1-D correlation matrix (symmetric eigendecomposition,
eigenvalues clipped at zero) and xi i.i.d. N(0,1) from a seeded generator:
an exact sample, computed with three 1-D contractions.

Output layout [E][qz][qy][qx], element index (ez*ny + ey)*nx + ex, as the
C ABI expects.
"""
from __future__ import annotations

import numpy as np


def gauss_points(n):
    if n == 1:
        return np.array([0.0])
    if n == 2:
        a = 1 / np.sqrt(3.0)
        return np.array([-a, a])
    if n == 3:
        a = np.sqrt(3 / 5)
        return np.array([-a, 0.0, a])
    a = np.sqrt(3 / 7 - 2 / 7 * np.sqrt(6 / 5))
    b = np.sqrt(3 / 7 + 2 / 7 * np.sqrt(6 / 5))
    return np.array([-b, -a, a, b])


def _factor_1d(coords, ell):
    d = coords[:, None] - coords[None, :]
    K = np.exp(-(d * d) / (2.0 * ell * ell))
    w, V = np.linalg.eigh(K)
    w = np.clip(w, 0.0, None)
    return V * np.sqrt(w)[None, :]


def qp_coords_1d(n_elem, nq):
    g = gauss_points(nq)
    return ((np.arange(n_elem)[:, None] + 0.5 * (1.0 + g[None, :])) / n_elem).ravel()


def gaussian_field_q(nx, ny, nz, nq, sigma2=1.0, ell=0.1, seed=0):
    rng = np.random.default_rng(seed)
    X, Y, Z = nx * nq, ny * nq, nz * nq
    Lx = _factor_1d(qp_coords_1d(nx, nq), ell)
    Ly = _factor_1d(qp_coords_1d(ny, nq), ell)
    Lz = _factor_1d(qp_coords_1d(nz, nq), ell)
    g = rng.standard_normal((Z, Y, X))
    g = g @ Lx.T                               # contract x
    g = np.matmul(Ly, g)                       # contract y (batched over z)
    g = (Lz @ g.reshape(Z, Y * X)).reshape(Z, Y, X)  # contract z
    g *= np.sqrt(sigma2)
    # (ez,qz,ey,qy,ex,qx) -> [E][qz][qy][qx]
    g = g.reshape(nz, nq, ny, nq, nx, nq).transpose(0, 2, 4, 1, 3, 5)
    return np.ascontiguousarray(g).reshape(-1)


def gaussian_field_q_torch(nx, ny, nz, nq, sigma2=1.0, ell=0.1, seed=0, device="cuda"):
    """Same construction as gaussian_field_q with the three contractions and
    the normal draws on a torch device (seeded torch generator), returned as a
    host float64 array in the [E][qz][qy][qx] layout."""
    import torch

    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    X, Y, Z = nx * nq, ny * nq, nz * nq
    Lx = torch.from_numpy(_factor_1d(qp_coords_1d(nx, nq), ell)).to(device)
    Ly = torch.from_numpy(_factor_1d(qp_coords_1d(ny, nq), ell)).to(device)
    Lz = torch.from_numpy(_factor_1d(qp_coords_1d(nz, nq), ell)).to(device)
    g = torch.randn((Z, Y, X), generator=gen, dtype=torch.float64, device=device)
    g = g @ Lx.T
    g = torch.matmul(Ly, g)
    g = (Lz @ g.reshape(Z, Y * X)).reshape(Z, Y, X)
    g *= float(np.sqrt(sigma2))
    g = g.reshape(nz, nq, ny, nq, nx, nq).permute(0, 2, 4, 1, 3, 5).contiguous()
    return g.reshape(-1).cpu().numpy()


def lognormal_kappa_q(nx, ny, nz, p, sigma2=1.0, ell=0.1, seed=0, device=None):
    """kappa = exp(g) at the quadrature points; device="cuda" draws on the GPU
    (a different, equally seeded stream of normals than the numpy path)."""
    if device is not None:
        g = gaussian_field_q_torch(nx, ny, nz, p + 1, sigma2, ell, seed, device)
    else:
        g = gaussian_field_q(nx, ny, nz, p + 1, sigma2, ell, seed)
    np.exp(g, out=g)
    return g


def sin_nodal(nx, ny, nz, p, scale=1.0):
    """f = 3 pi^2 sin(pi x) sin(pi y) sin(pi z) at the nodes of the unit-cube DOF grid."""
    xs = np.linspace(0.0, 1.0, nx * p + 1)
    ys = np.linspace(0.0, 1.0, ny * p + 1)
    zs = np.linspace(0.0, 1.0, nz * p + 1)
    s = 3.0 * np.pi ** 2 * scale
    return (s * np.sin(np.pi * zs)[:, None, None] * np.sin(np.pi * ys)[None, :, None]
            * np.sin(np.pi * xs)[None, None, :]).ravel()
