"""FP32 chosen form: the FP32 apply and FP32-apply/FP64-refinement PCG.

Tolerances, written here because the FP32 path is not bit-comparable:
  * FP32 apply vs the FP64 oracle: relative 2-norm error <= 2e-5 (FP32 rounding
    of the quadrature data and of ~1.5k FMAs per element);
  * FP32 mixed-precision solve (FP32 iterates, FP64 reliable updates): FP64 true relative residual <= 1e-8 (the solver's own
    target, recomputed in FP64) and relative error against the FP64 oracle
    solution <= 1e-7, for every result.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import femgpu  # noqa: E402
from femgpu.fields import lognormal_kappa_q  # noqa: E402

APPLY_TOL = 2e-5


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def apply_f32(op, x, constrained):
    x32 = np.ascontiguousarray(x, dtype=np.float32)
    y32 = np.zeros_like(x32)
    rc = femgpu.lib().fg_op_apply_f32(op.handle, x32.ctypes.data, y32.ctypes.data, 0, int(constrained),
                                      femgpu.HOST)
    assert rc == 0, femgpu.last_error()
    return y32.astype(np.float64)


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("kind", [femgpu.MASS, femgpu.DIFF, femgpu.MASS_DIFF])
def test_fp32_apply_matches_fp64_oracle(p, kind):
    need_gpu()
    nx, ny, nz = (37, 9, 10) if p < 3 else (33, 3, 4)
    rng = np.random.default_rng(p + 10 * kind)
    kq = np.exp(rng.normal(size=nx * ny * nz * (p + 1) ** 3))
    mesh = O.Mesh(nx, ny, nz, p)
    coef = O.Coef(kind, c_m=1.5, c_k=0.5, kappa_q=kq, rho=2.0)
    op = femgpu.PAOperator((nx, ny, nz), p, kind, kappa=kq, rho=2.0, c_mass=1.5, c_diff=0.5)
    x = rng.normal(size=mesh.ndofs)
    for constrained in (False, True):
        y = apply_f32(op, x, constrained)
        ref = (O.apply_constrained(mesh, coef, O.ess_mask(mesh), x) if constrained
               else O.pa_apply(mesh, coef, x))
        err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
        assert err <= APPLY_TOL, err


@pytest.mark.parametrize("precond", [femgpu.PC_JACOBI, femgpu.PC_CHEBYSHEV])
@pytest.mark.parametrize("p", [1, 2])
def test_fp32_ir_solve_reaches_fp64_residual(p, precond):
    need_gpu()
    n = {1: 20, 2: 12}[p]
    kq = lognormal_kappa_q(n, n, n, p, sigma2=1.0, ell=0.1, seed=3)
    mesh = O.Mesh(n, n, n, p)
    mask = O.ess_mask(mesh)
    coef = O.Coef(O.DIFF, kappa_q=kq)
    b = O.source(mesh, mask)
    x_ref, _ = O.pcg(mesh, coef, mask, b, precond=1, rtol=1e-13, max_iter=20000)
    op = femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
    cfg64 = femgpu.SolverConfig(rtol=1e-8, max_iter=20000)
    x64 = np.zeros(mesh.ndofs)
    r64 = op.pcg(b, x64, cfg64, precond)
    cfg32 = femgpu.SolverConfig(rtol=1e-8, max_iter=20000, precision=femgpu.FP32_IR)
    x32 = np.zeros(mesh.ndofs)
    r32 = op.pcg(b, x32, cfg32, precond)
    assert r64.converged and r32.converged
    assert r32.true_residual <= 1e-8, r32.true_residual
    assert r32.outer_iterations >= 1  # FP64 reliable updates happened
    err32 = np.linalg.norm(x32 - x_ref) / np.linalg.norm(x_ref)
    err64 = np.linalg.norm(x64 - x_ref) / np.linalg.norm(x_ref)
    assert err32 <= 1e-7, (err32, err64)
    # reliable updates keep the Krylov space: iterations stay close to plain FP64
    assert r32.iterations <= 1.2 * r64.iterations + 5, (r32.iterations, r64.iterations)
