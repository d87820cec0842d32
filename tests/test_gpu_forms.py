"""One-time work around the solve on the GPU, against the oracle:
Gauss-point coordinates, the source linear form (DomainSourceIntegrator +
assemble_linear, standard/source.rs:39-50), the L2 error of
examples/mfem_ex1_poisson.rs:119-162 and the lumped mass operator
(partial.rs:217-274).  Tolerance 1e-12 relative (FP64, different summation
order); the mfem_ex1 known answers (L2 < 2.2e-2 at n = 8, rate > 1.5) are
reproduced with every step on the GPU."""
import numpy as np
import pytest

from conftest import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import femgpu  # noqa: E402


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


def perturbed_vertices(nx, ny, nz, seed, amp=0.2):
    v = femgpu.unit_cube_vertices(nx, ny, nz).reshape(nz + 1, ny + 1, nx + 1, 3)
    rng = np.random.default_rng(seed)
    h = np.array([1 / nx, 1 / ny, 1 / nz])
    v[1:-1, 1:-1, 1:-1] += amp * h * rng.uniform(-1, 1, size=v[1:-1, 1:-1, 1:-1].shape)
    return v.reshape(-1, 3)


def trilinear_points(nx, ny, nz, vc, nq):
    xg, _ = np.polynomial.legendre.leggauss(nq)
    V = vc.reshape(nz + 1, ny + 1, nx + 1, 3)
    out = np.zeros((nx * ny * nz, nq ** 3, 3))
    for e in range(nx * ny * nz):
        ex, ey, ez = e % nx, (e // nx) % ny, e // (nx * ny)
        q = 0
        for kz in range(nq):
            for ky in range(nq):
                for kx in range(nq):
                    s = np.zeros(3)
                    for dz in (0, 1):
                        for dy in (0, 1):
                            for dx in (0, 1):
                                wgt = ((1 + (2 * dx - 1) * xg[kx]) * (1 + (2 * dy - 1) * xg[ky])
                                       * (1 + (2 * dz - 1) * xg[kz])) / 8
                                s += wgt * V[ez + dz, ey + dy, ex + dx]
                    out[e, q] = s
                    q += 1
    return out


def f_sin(xyz):
    return 3 * np.pi ** 2 * np.prod(np.sin(np.pi * xyz), axis=-1)


def u_sin(xyz):
    return np.prod(np.sin(np.pi * xyz), axis=-1)


@pytest.mark.parametrize("nq", [2, 3, 5])
def test_quadrature_points(nq):
    need_gpu()
    nx, ny, nz = 3, 2, 4
    vc = perturbed_vertices(nx, ny, nz, 1)
    got = femgpu.quadrature_points(nx, ny, nz, nq, vc)
    assert np.abs(got - trilinear_points(nx, ny, nz, vc, nq)).max() < 1e-14
    got_u = femgpu.quadrature_points(nx, ny, nz, nq)
    ref_u = trilinear_points(nx, ny, nz, femgpu.unit_cube_vertices(nx, ny, nz), nq)
    assert np.abs(got_u - ref_u).max() < 1e-14


@pytest.mark.parametrize("p", [1, 2, 3])
def test_source_matches_oracle(p):
    need_gpu()
    nx, ny, nz = 5, 4, 3
    vc = perturbed_vertices(nx, ny, nz, 2)
    mesh = O.Mesh(nx, ny, nz, p, vcoord=vc)
    mask = O.ess_mask(mesh)
    fq = f_sin(femgpu.quadrature_points(nx, ny, nz, p + 1, vc))
    b = femgpu.assemble_source(nx, ny, nz, p, fq, vcoord=vc)
    assert rel(b, O.source(mesh, mask)) <= 1e-12
    # no essential rows, constant f: the row sums of the mass matrix
    b1 = femgpu.assemble_source(nx, ny, nz, p, None, f=2.5, ess_tags=0, vcoord=vc)
    m1 = O.pa_apply(mesh, O.Coef(O.MASS, rho=2.5), np.ones(mesh.ndofs))
    assert rel(b1, m1) <= 1e-12


@pytest.mark.parametrize("p", [1, 2, 3])
def test_l2_error_matches_oracle(p):
    need_gpu()
    nx, ny, nz = 4, 3, 5
    vc = perturbed_vertices(nx, ny, nz, 3)
    mesh = O.Mesh(nx, ny, nz, p, vcoord=vc)
    u = np.random.default_rng(4).standard_normal(mesh.ndofs)
    nq = min(p + 2, 4)  # the oracle's rules (hex_rule) have at most 4 points
    uq = u_sin(femgpu.quadrature_points(nx, ny, nz, nq, vc))
    e = femgpu.l2_error(nx, ny, nz, p, u, uq, nq=nq, vcoord=vc)
    assert abs(e - O.l2_error_sin(mesh, u, nq=nq)) <= 1e-12 * e


@pytest.mark.parametrize("p", [1, 2, 3])
def test_lumped_mass_matches_oracle(p):
    need_gpu()
    nx, ny, nz = 3, 4, 2
    vc = perturbed_vertices(nx, ny, nz, 5)
    mesh = O.Mesh(nx, ny, nz, p, vcoord=vc)
    rq = np.exp(np.random.default_rng(6).normal(size=mesh.n_elem * (p + 1) ** 3))
    lm = femgpu.LumpedMassOperator(nx, ny, nz, p, rho_q=rq, vcoord=vc)
    assert rel(lm.diag, O.lumped_mass(mesh, rq)) <= 1e-12
    lc = femgpu.LumpedMassOperator(nx, ny, nz, p, rho=1.7, vcoord=vc)
    assert rel(lc.diag, O.lumped_mass(mesh, None, 1.7)) <= 1e-12
    # total mass = rho |Omega| (standard/mass.rs:67-82 on the lumped form)
    vol = O.lumped_mass(mesh, None, 1.0).sum()
    assert abs(lc.diag.sum() - 1.7 * vol) <= 1e-12 * vol
    x = np.random.default_rng(7).standard_normal(len(lm.diag))
    y = np.ones_like(x)
    lm.apply(x, y)  # the device may fuse the multiply-add (one rounding)
    assert np.allclose(y, 1.0 + lm.diag * x, rtol=1e-15, atol=0)
    lm.apply_zero(x, y)
    assert np.array_equal(y, lm.diag * x)
    lm.apply_inverse(x, y)
    assert np.allclose(y, x / lm.diag, rtol=1e-15, atol=0)
    # zero-length vectors are a no-op (no launch)
    empty = np.zeros(0)
    assert femgpu.lib().fg_lumped_apply(lm.diag.ctypes.data, empty.ctypes.data, empty.ctypes.data, 0, 0,
                                        femgpu.HOST) == 0


def test_ex1_known_answers_on_gpu():
    """mfem_ex1_poisson.rs:184-208: L2 < 2.2e-2 at n = 8 (Q1) and rate > 1.5,
    source, solve and error all on the GPU."""
    need_gpu()
    errs = []
    for n in (8, 16):
        op = femgpu.PADiffusionOperator((n, n, n), 1)
        b = femgpu.assemble_source(n, n, n, 1, f_sin(femgpu.quadrature_points(n, n, n, 2)))
        x = np.zeros(op.n_dofs())
        r = femgpu.solve_pcg_jacobi(op, b, x, femgpu.SolverConfig(rtol=1e-10, max_iter=2000))
        assert r.converged
        errs.append(femgpu.l2_error(n, n, n, 1, x, u_sin(femgpu.quadrature_points(n, n, n, 3)), nq=3))
        op.close()
    assert errs[0] < 2.2e-2
    assert np.log2(errs[0] / errs[1]) > 1.5


def test_forms_reject_bad_arguments():
    need_gpu()
    with pytest.raises(femgpu.SolverError):
        femgpu.quadrature_points(2, 2, 2, 9)
    with pytest.raises(femgpu.SolverError):
        femgpu.assemble_source(2, 2, 2, 4)
    with pytest.raises(femgpu.SolverError):
        femgpu.l2_error(2, 2, 2, 1, np.zeros(27), nq=9)
