"""Affine-compressed quadrature data (fg_op_set_qdata_format(FG_QDATA_AFFINE)).

On meshes whose elements have a constant Jacobian (uniform boxes and their
affine images) the compressed format must reproduce the oracle apply with the
same tolerances as the full format: 1e-12 relative in FP64, 2e-5 in FP32.  On
a non-affine mesh the format must be refused (FG_UNSUPPORTED) and the handle
keep working in the full format.
"""
import numpy as np
import pytest

from conftest import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import femgpu  # noqa: E402


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def sheared_vertices(nx, ny, nz):
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    v = np.stack([i / nx, j / ny, k / nz], axis=-1).reshape(-1, 3).astype(np.float64)
    A = np.array([[1.2, 0.3, -0.1], [0.0, 0.9, 0.25], [0.1, -0.2, 1.1]])
    return v @ A.T + np.array([0.3, -0.2, 0.5])


def f32_apply(op, x, constrained):
    x32 = np.ascontiguousarray(x, dtype=np.float32)
    y32 = np.zeros_like(x32)
    rc = femgpu.lib().fg_op_apply_f32(op.handle, x32.ctypes.data, y32.ctypes.data, 0, int(constrained), femgpu.HOST)
    assert rc == 0, femgpu.last_error()
    return y32.astype(np.float64)


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("kind", [femgpu.MASS, femgpu.DIFF, femgpu.MASS_DIFF])
@pytest.mark.parametrize("sheared", [False, True])
def test_affine_format_matches_oracle(p, kind, sheared):
    need_gpu()
    nx, ny, nz = (35, 6, 9) if p < 3 else (33, 3, 3)
    vc = sheared_vertices(nx, ny, nz) if sheared else None
    rng = np.random.default_rng(p * 7 + kind)
    kq = np.exp(rng.normal(size=nx * ny * nz * (p + 1) ** 3))
    rq = np.exp(0.2 * rng.normal(size=kq.size))
    mesh = O.Mesh(nx, ny, nz, p, vcoord=vc)
    coef = O.Coef(kind, c_m=0.7, c_k=1.3, kappa_q=kq, rho_q=rq)
    op = femgpu.PAOperator(dict(nx=nx, ny=ny, nz=nz, vcoord=vc), p, kind, kappa=kq, rho=rq,
                           c_mass=0.7, c_diff=1.3)
    x = rng.normal(size=mesh.ndofs)
    y_full = op.matvec(x)
    op.set_qdata_format(femgpu.QDATA_AFFINE)
    for constrained in (False, True):
        ref = (O.apply_constrained(mesh, coef, O.ess_mask(mesh), x) if constrained else O.pa_apply(mesh, coef, x))
        y = op.matvec(x, constrained=constrained)
        assert np.linalg.norm(y - ref) <= 1e-12 * np.linalg.norm(ref)
        y32 = f32_apply(op, x, constrained)
        assert np.linalg.norm(y32 - ref) <= 2e-5 * np.linalg.norm(ref)
    op.set_qdata_format(femgpu.QDATA_FULL)
    assert np.array_equal(op.matvec(x), y_full)


def test_affine_format_refused_on_distorted_mesh():
    need_gpu()
    nx = ny = nz = 4
    rng = np.random.default_rng(0)
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    v = np.stack([i / nx, j / ny, k / nz], axis=-1).astype(np.float64)
    v[2, 2, 2] += 0.05
    op = femgpu.PADiffusionOperator(dict(nx=nx, ny=ny, nz=nz, vcoord=v.reshape(-1, 3)), 2)
    x = rng.normal(size=op.n_dofs())
    y = op.matvec(x)
    with pytest.raises(femgpu.SolverError) as ei:
        op.set_qdata_format(femgpu.QDATA_AFFINE)
    assert ei.value.status == femgpu.FG_UNSUPPORTED
    assert np.array_equal(op.matvec(x), y)


def test_affine_fp32_solve_meets_fp64_target():
    need_gpu()
    from femgpu.fields import lognormal_kappa_q
    n, p = 12, 2
    kq = lognormal_kappa_q(n, n, n, p, seed=5)
    mesh = O.Mesh(n, n, n, p)
    mask = O.ess_mask(mesh)
    coef = O.Coef(O.DIFF, kappa_q=kq)
    b = O.source(mesh, mask)
    x_ref, _ = O.pcg(mesh, coef, mask, b, precond=1, rtol=1e-13, max_iter=20000)
    op = femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
    op.set_qdata_format(femgpu.QDATA_AFFINE)
    for pc in (femgpu.PC_JACOBI, femgpu.PC_CHEBYSHEV):
        x = np.zeros(mesh.ndofs)
        r = op.pcg(b, x, femgpu.SolverConfig(rtol=1e-8, max_iter=5000, precision=femgpu.FP32_IR), pc)
        assert r.converged and r.true_residual <= 1e-8
        assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) <= 1e-7
