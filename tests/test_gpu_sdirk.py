"""SDIRK-2 heat stepping on the GPU (fg_sdirk2) against an SDIRK-2 loop driven
by the oracle (the stage systems of examples/mfem_ex10_heat_equation.rs:201-250
with the oracle's PCG and constrained apply), plus the reference example's own
checks: error against the exact decaying mode and sign symmetry
(mfem_ex10_heat_equation.rs:379-420).
"""
import math

import numpy as np
import pytest

from conftest import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import femgpu  # noqa: E402
from femgpu.fields import lognormal_kappa_q  # noqa: E402

G = femgpu.SDIRK2_GAMMA


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def initial(n, p, scale=1.0):
    xs = np.linspace(0, 1, n * p + 1)
    u = scale * (np.sin(np.pi * xs)[:, None, None] * np.sin(np.pi * xs)[None, :, None]
                 * np.sin(np.pi * xs)[None, None, :]).ravel()
    return u


def oracle_sdirk(mesh, kq, u, dt, steps):
    mask = O.ess_mask(mesh)
    u = u.copy()
    u[mask == 1] = 0.0
    K = O.Coef(O.DIFF, kappa_q=kq)
    S = O.Coef(O.MASS_DIFF, c_m=1.0, c_k=G * dt, kappa_q=kq)
    for _ in range(steps):
        rhs = -O.apply_constrained(mesh, K, mask, u)
        k1, _ = O.pcg(mesh, S, mask, rhs, precond=1, rtol=1e-13, max_iter=5000)
        u2 = u + dt * (1 - G) * k1
        rhs = -O.apply_constrained(mesh, K, mask, u2)
        k2, _ = O.pcg(mesh, S, mask, rhs, precond=1, rtol=1e-13, max_iter=5000)
        u = u + dt * ((1 - G) * k1 + G * k2)
    return u


def make_ops(n, p, kq, dt):
    K = femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
    S = femgpu.PAMassDiffusionOperator((n, n, n), p, 1.0, G * dt, kappa=kq)
    return K, S


def test_sdirk_matches_oracle_driven_loop():
    need_gpu()
    n, p, dt, steps = 6, 2, 1e-3, 4
    kq = lognormal_kappa_q(n, n, n, p, seed=2)
    mesh = O.Mesh(n, n, n, p)
    u0 = initial(n, p)
    u0[O.ess_mask(mesh) == 1] = 0.0
    ref = oracle_sdirk(mesh, kq, u0, dt, steps)
    K, S = make_ops(n, p, kq, dt)
    u = u0.copy()
    info = femgpu.sdirk2(K, S, u, dt, steps, femgpu.SolverConfig(rtol=1e-13, max_iter=5000))
    assert info["steps"] == steps and info["total_iterations"] > 0
    assert np.linalg.norm(u - ref) <= 1e-10 * np.linalg.norm(ref)


def test_sdirk_decay_accuracy_and_sign_symmetry():
    """ex10: coarse SDIRK-2 error small; negated initial data negates the solution."""
    need_gpu()
    n, p, dt, t_end = 8, 2, 0.01, 0.1
    steps = int(round(t_end / dt))
    K, S = make_ops(n, p, 1.0, dt)
    mesh = O.Mesh(n, n, n, p)
    mask = O.ess_mask(mesh)
    up = initial(n, p)
    up[mask == 1] = 0.0
    un = -up
    cfg = femgpu.SolverConfig(rtol=1e-12, max_iter=5000)
    femgpu.sdirk2(K, S, up, dt, steps, cfg)
    femgpu.sdirk2(K, S, un, dt, steps, cfg)
    exact = math.exp(-3 * math.pi ** 2 * t_end) * initial(n, p)
    exact[mask == 1] = 0.0
    rms = np.sqrt(np.mean((up - exact) ** 2))
    assert rms < 5e-3, rms
    assert abs(np.linalg.norm(up) - np.linalg.norm(un)) < 1e-12
    assert np.abs(up + un).max() < 1e-12


@pytest.mark.parametrize("precond", [femgpu.PC_JACOBI, femgpu.PC_CHEBYSHEV])
def test_sdirk_fp32_stages_match_fp64(precond):
    need_gpu()
    n, p, dt, steps = 10, 2, 1e-3, 6
    kq = lognormal_kappa_q(n, n, n, p, seed=4)
    K, S = make_ops(n, p, kq, dt)
    mesh = O.Mesh(n, n, n, p)
    u0 = initial(n, p)
    u0[O.ess_mask(mesh) == 1] = 0.0
    u64, u32 = u0.copy(), u0.copy()
    femgpu.sdirk2(K, S, u64, dt, steps, femgpu.SolverConfig(rtol=1e-10), precond)
    femgpu.sdirk2(K, S, u32, dt, steps, femgpu.SolverConfig(rtol=1e-10, precision=femgpu.FP32_IR), precond)
    assert np.linalg.norm(u32 - u64) <= 1e-7 * np.linalg.norm(u64)


@pytest.mark.parametrize("prec", [femgpu.FP64, femgpu.FP32_IR])
def test_sdirk_affine_qdata_matches_full(prec):
    """Both stage operators in the affine-compressed quadrature-data format
    (uniform mesh: constant J per element, kappa per point) give the FP64
    full-format trajectory to 1e-7 (FP32 stages) / 1e-10 (FP64 stages)."""
    need_gpu()
    n, p, dt, steps = 10, 2, 1e-3, 6
    kq = lognormal_kappa_q(n, n, n, p, seed=5)
    K, S = make_ops(n, p, kq, dt)
    mesh = O.Mesh(n, n, n, p)
    u0 = initial(n, p)
    u0[O.ess_mask(mesh) == 1] = 0.0
    ref, u = u0.copy(), u0.copy()
    femgpu.sdirk2(K, S, ref, dt, steps, femgpu.SolverConfig(rtol=1e-12), femgpu.PC_CHEBYSHEV)
    K.set_qdata_format(femgpu.QDATA_AFFINE)
    S.set_qdata_format(femgpu.QDATA_AFFINE)
    femgpu.sdirk2(K, S, u, dt, steps, femgpu.SolverConfig(rtol=1e-12, precision=prec), femgpu.PC_CHEBYSHEV)
    tol = 1e-10 if prec == femgpu.FP64 else 1e-7
    assert np.linalg.norm(u - ref) <= tol * np.linalg.norm(ref)


@pytest.mark.parametrize("prec", [femgpu.FP64, femgpu.FP32_IR])
def test_sdirk_survives_strong_decay(prec):
    """The stage right-hand sides shrink with the solution (here by ~1e-120);
    stage solves on normalised right-hand sides must still all converge."""
    need_gpu()
    n, p, dt, steps = 5, 2, 1e-3, 200
    K, S = make_ops(n, p, 50.0, dt)
    mesh = O.Mesh(n, n, n, p)
    u = initial(n, p)
    u[O.ess_mask(mesh) == 1] = 0.0
    info = femgpu.sdirk2(K, S, u, dt, steps, femgpu.SolverConfig(rtol=1e-10, precision=prec), femgpu.PC_CHEBYSHEV)
    assert info["steps"] == steps
    assert np.all(np.isfinite(u)) and np.abs(u).max() < 1e-100
