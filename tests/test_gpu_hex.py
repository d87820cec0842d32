"""The unstructured Hex8 operator (fg_op_create_hex) against the oracle.

The drop-in case: a caller holding a Hex8 mesh and a DofManager numbering.
Here that mesh is a perturbed box (so the oracle's structured element loop
gives the answer) handed over with every numbering scrambled:

* nodes, DOFs and elements in random order;
* each element's local frame changed by a random symmetry of the reference
  cube (axis permutation and reflections): its 8 vertices in HexQ1 order
  (crates/element/src/lagrange/hex.rs:27-36), its DOF map in the tensor order
  of the new frame and its kappa table at the new frame's Gauss points all
  follow.  The Gauss rule is invariant under these symmetries, so the operator
  is unchanged up to rounding;
* an arbitrary essential-DOF list (two boundary faces and random interior
  DOFs), the form boundary_dofs returns (crates/space/src/constraints.rs:53-60).

Tolerances: 1e-12 relative for the FP64 apply and diagonal (the north-star
bar); Jacobi-PCG iterations within +-1 of the oracle's
(crates/parallel/src/par_solver.rs:262-342).
"""
import itertools

import numpy as np
import pytest

from conftest import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import femgpu  # noqa: E402

RTOL = 1e-12
HEXQ1 = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
SYMS = [(perm, flip) for perm in itertools.permutations(range(3)) for flip in itertools.product((0, 1), repeat=3)]


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def relerr(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def perturbed_vertices(nx, ny, nz, amp, rng):
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    v = np.stack([i / nx, j / ny, k / nz], axis=-1).astype(np.float64)
    inner = (i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)
    v[inner] += amp * np.array([1 / nx, 1 / ny, 1 / nz]) * rng.uniform(-1, 1, size=(inner.sum(), 3))
    return v.reshape(-1, 3)


def scrambled_mesh(nx, ny, nz, p, kq, seed):
    """The box (nx, ny, nz) of order p as an unstructured Hex8 mesh with random
    node / DOF / element numbering and a random reference-frame symmetry per
    element.  Returns the arrays of fg_op_create_hex (element DOF maps in the
    tensor order of the new frame, or in HexQ1 vertex order for p = 1), the
    node and DOF permutations (new id of box vertex / DOF d) and the kappa
    table at the new frames' Gauss points."""
    rng = np.random.default_rng(seed)
    q = p + 1
    NI, NJ, NK = nx * p + 1, ny * p + 1, nz * p + 1
    n_nodes = (nx + 1) * (ny + 1) * (nz + 1)
    N = NI * NJ * NK
    pn = rng.permutation(n_nodes)  # box vertex -> new node id
    pd = rng.permutation(N)        # box DOF -> new DOF id
    pe = rng.permutation(nx * ny * nz)  # new element -> box element
    E = pe.size
    conn = np.zeros((E, 8), dtype=np.uint32)
    ed = np.zeros((E, q ** 3), dtype=np.uint32)
    kq_new = None if kq is None else np.zeros((E, q ** 3))
    for s, e in enumerate(pe):
        ex, ey, ez = e % nx, (e // nx) % ny, e // (nx * ny)
        perm, flip = SYMS[rng.integers(len(SYMS))]

        def orig(u, m):  # new-frame tensor index u (entries 0..m) -> box-frame index
            t = [0, 0, 0]
            for d in range(3):
                t[perm[d]] = m - u[d] if flip[d] else u[d]
            return t

        for h, u in enumerate(HEXQ1):
            t = orig(u, 1)
            conn[s, h] = pn[((ez + t[2]) * (ny + 1) + ey + t[1]) * (nx + 1) + ex + t[0]]
        for c, b, a in itertools.product(range(q), repeat=3):
            k = (c * q + b) * q + a
            t = orig((a, b, c), p)
            ed[s, k] = pd[((ez * p + t[2]) * NJ + ey * p + t[1]) * NI + ex * p + t[0]]
            if kq is not None:
                kq_new[s, k] = kq[e * q ** 3 + (t[2] * q + t[1]) * q + t[0]]
    if p == 1:  # order-1 element DOF maps are given in the HexQ1 vertex order
        ed = np.ascontiguousarray(ed[:, [(c * 2 + b) * 2 + a for a, b, c in HEXQ1]])
    return conn, ed, pn, pd, kq_new


def _coords(vc, pn):
    out = np.zeros_like(vc)
    out[pn] = vc
    return out


@pytest.mark.parametrize("p,shape", [(1, (9, 7, 6)), (2, (7, 5, 6)), (3, (5, 4, 4)),
                                     (1, (20, 16, 13)), (2, (13, 11, 9)), (3, (9, 8, 7))])
@pytest.mark.parametrize("kind", [femgpu.DIFF, femgpu.MASS_DIFF])
def test_scrambled_hex_mesh_matches_oracle(p, shape, kind):
    """Scrambled element order and DOF numbering, perturbed vertices, an
    arbitrary essential list; the larger meshes span many element chunks, so
    most DOFs on chunk borders go through the shared-DOF partials."""
    need_gpu()
    nx, ny, nz = shape
    rng = np.random.default_rng(10 * p + kind)
    vc = perturbed_vertices(nx, ny, nz, 0.2, rng)
    kq = np.exp(rng.normal(size=nx * ny * nz * (p + 1) ** 3))
    mesh = O.Mesh(nx, ny, nz, p, vcoord=vc)
    coef = O.Coef(kind, c_m=0.7, c_k=1.3, kappa_q=kq)
    conn, ed, pn, pd, kq_new = scrambled_mesh(nx, ny, nz, p, kq, seed=p)
    N = mesh.ndofs
    # essential DOFs: faces x0 and z1 of the box plus 5 % random DOFs
    mask = O.ess_mask(mesh, 16 | 2).astype(bool)
    mask[rng.random(N) < 0.05] = True
    ess_new = pd[np.flatnonzero(mask)]
    ess_new = np.concatenate([ess_new, ess_new[:7]])  # repeats are allowed
    rng.shuffle(ess_new)
    op = femgpu.HexMeshOperator(p, _coords(vc, pn), conn, elem_dofs=ed, n_dofs=N, kind=kind, kappa=kq_new,
                                c_mass=0.7, c_diff=1.3, ess_dofs=ess_new)
    assert op.n_dofs() == N and op.chunks == -(-nx * ny * nz // (128 if p < 3 else 64))
    x = rng.standard_normal(N)
    xn = np.zeros(N)
    xn[pd] = x
    # raw and constrained apply, the accumulate form, the diagonal
    y = op.matvec(xn)[pd]
    assert relerr(y, O.pa_apply(mesh, coef, x)) <= RTOL
    m8 = mask.astype(np.uint8)
    yc_ref = O.apply_constrained(mesh, coef, m8, x)
    yc = op.matvec(xn, constrained=True)
    assert relerr(yc[pd], yc_ref) <= RTOL
    y2 = yc.copy()
    op.apply(xn, y2, constrained=True)
    assert relerr(y2[pd], 2 * yc_ref) <= RTOL
    d = op.diagonal(constrained=True)[pd]
    assert relerr(d, O.diagonal(mesh, coef, m8)) <= RTOL
    # bit-for-bit repeatable
    assert np.array_equal(op.matvec(xn, constrained=True), yc)
    op.close()


@pytest.mark.parametrize("p", [1, 2])
def test_scrambled_hex_mesh_pcg(p):
    """Jacobi-PCG iterations within +-1 of the oracle's on the scrambled mesh;
    Chebyshev and FP32-in-FP64 solves reach the FP64 target and agree with the
    oracle's solution."""
    need_gpu()
    nx, ny, nz = (14, 12, 10) if p == 1 else (8, 7, 6)
    rng = np.random.default_rng(77 + p)
    vc = perturbed_vertices(nx, ny, nz, 0.15, rng)
    kq = np.exp(rng.normal(size=nx * ny * nz * (p + 1) ** 3))
    mesh = O.Mesh(nx, ny, nz, p, vcoord=vc)
    coef = O.Coef(O.DIFF, kappa_q=kq)
    mask = O.ess_mask(mesh, 63).astype(bool)
    mask[rng.random(mesh.ndofs) < 0.02] = True
    m8 = mask.astype(np.uint8)
    b = rng.standard_normal(mesh.ndofs)
    b[mask] = 0.0
    x_ref, info = O.pcg(mesh, coef, m8, b, precond=1, rtol=1e-10, max_iter=5000)
    assert info["converged"] and info["iterations"] > 30
    conn, ed, pn, pd, kq_new = scrambled_mesh(nx, ny, nz, p, kq, seed=5 + p)
    # order 1: DOF = node, no element DOF maps (DofManager::build_p1)
    if p == 1:
        relabel = np.zeros(mesh.ndofs, dtype=np.uint32)
        relabel[pn] = pd      # new node id -> new DOF id ...
        conn = relabel[conn]  # ... so that DOF = node in the handed-over mesh
        coords = np.zeros_like(vc)
        coords[pd] = vc
        op = femgpu.HexMeshOperator(1, coords, conn, kappa=kq_new, ess_dofs=pd[np.flatnonzero(mask)])
    else:
        op = femgpu.HexMeshOperator(p, _coords(vc, pn), conn, elem_dofs=ed, n_dofs=mesh.ndofs, kappa=kq_new,
                                    ess_dofs=pd[np.flatnonzero(mask)])
    bn = np.zeros(mesh.ndofs)
    bn[pd] = b
    x = np.zeros(mesh.ndofs)
    res = femgpu.solve_pcg_jacobi(op, bn, x, femgpu.SolverConfig(rtol=1e-10, max_iter=5000))
    assert res.converged and abs(res.iterations - info["iterations"]) <= 1, (res.iterations, info["iterations"])
    assert relerr(x[pd], x_ref) < 1e-7
    for prec in (femgpu.FP64, femgpu.FP32_IR):
        x = np.zeros(mesh.ndofs)
        r = op.pcg(bn, x, femgpu.SolverConfig(rtol=1e-8, max_iter=5000, precision=prec), femgpu.PC_CHEBYSHEV)
        assert r.converged and r.true_residual <= 1.05e-8
        assert relerr(x[pd], x_ref) < 1e-6
    op.close()


def test_hex_mesh_refuses_box_only_entry_points_and_bad_input():
    need_gpu()
    nx = ny = nz = 3
    conn, ed, pn, pd, _ = scrambled_mesh(nx, ny, nz, 2, None, seed=1)
    vc = _coords(perturbed_vertices(nx, ny, nz, 0.0, np.random.default_rng(0)), pn)
    op = femgpu.HexMeshOperator(2, vc, conn, elem_dofs=ed, n_dofs=7 ** 3)
    with pytest.raises(femgpu.SolverError) as exc:
        op.set_qdata_format(femgpu.QDATA_AFFINE)
    assert exc.value.status == femgpu.FG_UNSUPPORTED
    with pytest.raises(femgpu.SolverError):
        op.set_tile(2)
    op.close()
    bad = ed.copy()
    bad[3, 5] = 7 ** 3  # a DOF id past n_dofs
    with pytest.raises(femgpu.SolverError) as exc:
        femgpu.HexMeshOperator(2, vc, conn, elem_dofs=bad, n_dofs=7 ** 3)
    assert exc.value.status == femgpu.FG_BOUNDS
    flat = vc.copy()
    flat[:, 2] = 0.0  # every element collapsed onto z = 0
    with pytest.raises(femgpu.SolverError) as exc:
        femgpu.HexMeshOperator(2, flat, conn, elem_dofs=ed, n_dofs=7 ** 3)
    assert exc.value.status == femgpu.FG_BOUNDS
