"""fg_op_apply_native_noalloc: the apply for callers that cannot let the
library allocate device memory (their own pool owns the GPU memory, or they
cannot afford cudaMalloc's implicit synchronisation).  Its fix-up scratch is a
fixed 32 MiB array inside libfemgpu.so instead of a buffer the handle owns.

Checked here through the C ABI, for Q1, Q2 and Q3 (Q3 runs the slab kernel):
two calls in a row (different inputs; the array keeps the previous call's
contents) agree with fg_op_apply_native and with the oracle within the 1e-12
relative tolerance of the parity tests.  Before each case a differently
shaped operator with a larger face stride runs a noalloc apply on random
input, so the array holds non-zero data at offsets the case under test does
not use: a face slot the apply failed to write before the fix-up read it
would show up as a wrong result.  An operator whose face scratch exceeds the
array is rejected with a clear error.  This file is named to be collected
last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import femgpu  # noqa: E402

RTOL = 1e-12


def _lib():
    L = femgpu.lib()
    L.fg_op_apply_native_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
    L.fg_op_apply_native_noalloc.restype = C.c_int
    return L


def _vertices(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    v = np.stack([i / nx, j / ny, k / nz], axis=-1).astype(np.float64)
    inner = (i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)
    v[inner] += 0.1 * np.array([1 / nx, 1 / ny, 1 / nz]) * rng.uniform(-1, 1, size=(inner.sum(), 3))
    return v.reshape(-1, 3)


def _dirty_scratch(L, dev):
    """A noalloc apply of another operator (Q3 mass + diffusion, TZ 16: a
    larger face stride than the cases below) on random input, which leaves
    non-zero partials all over the static array."""
    op = femgpu.PAOperator((70, 9, 40), 3, femgpu.MASS_DIFF, c_mass=0.3)
    op.set_tile(16)
    x = torch.randn(op.native_len, dtype=torch.float64, device=dev)
    x.view(op.NK, op.NJ, op.NIp)[:, :, op.NI:] = 0.0
    y = torch.zeros_like(x)
    rc = L.fg_op_apply_native_noalloc(op.handle, x.data_ptr(), y.data_ptr(), 0, 0)
    assert rc == femgpu.FG_OK, femgpu.last_error()
    torch.cuda.synchronize()
    op.check()
    assert y.abs().max().item() > 0
    op.close()


@pytest.mark.parametrize("order,shape,kind", [(2, (40, 9, 17), femgpu.DIFF),
                                              (1, (70, 13, 20), femgpu.MASS_DIFF),
                                              (3, (37, 5, 11), femgpu.DIFF)])
def test_noalloc_apply_matches_regular_apply_and_oracle_twice(order, shape, kind):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = _lib()
    dev = torch.device("cuda", torch.cuda.current_device())
    _dirty_scratch(L, dev)
    nx, ny, nz = shape
    rng = np.random.default_rng(order)
    kq = np.exp(rng.normal(size=nx * ny * nz * (order + 1) ** 3))
    vc = _vertices(nx, ny, nz, order)
    op = femgpu.PAOperator(dict(nx=nx, ny=ny, nz=nz, vcoord=vc), order, kind,
                           kappa=kq, rho=2.0, c_mass=0.5, c_diff=1.5)
    mesh = O.Mesh(nx, ny, nz, order, vcoord=vc)
    coef = O.Coef(kind, c_m=0.5, c_k=1.5, kappa_q=kq, rho=2.0)
    mask = O.ess_mask(mesh)
    for call, seed in enumerate((11, 12)):
        xh = np.random.default_rng(seed).normal(size=op.n_dofs())
        x = torch.from_numpy(op.to_native(xh)).to(dev)
        y_ref = torch.zeros_like(x)
        y_new = torch.full_like(x, float("nan"))
        # pads of native vectors must hold zeros; real entries are all overwritten
        y_new.view(op.NK, op.NJ, op.NIp)[:, :, op.NI:] = 0.0
        op.apply_native(x.data_ptr(), y_ref.data_ptr(), accumulate=False, constrained=True)
        rc = L.fg_op_apply_native_noalloc(op.handle, x.data_ptr(), y_new.data_ptr(), 0, 1)
        assert rc == femgpu.FG_OK, femgpu.last_error()
        torch.cuda.synchronize()
        op.check()
        a, b = y_new.cpu().numpy(), y_ref.cpu().numpy()
        assert not np.isnan(a).any(), f"call {call}: unwritten entries"
        assert np.linalg.norm(a - b) <= RTOL * np.linalg.norm(b), f"call {call}"
        y_or = O.apply_constrained(mesh, coef, mask, xh)
        an = op.from_native(a)
        assert np.linalg.norm(an - y_or) <= RTOL * np.linalg.norm(y_or), f"call {call} vs oracle"
    op.close()


def test_noalloc_rejects_operator_larger_than_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = _lib()
    # 256 x 256 x 136 Q1 mass: 8704 tiles x 507 face doubles > 4 Mi doubles
    op = femgpu.PAOperator((256, 256, 136), 1, femgpu.MASS)
    x = torch.zeros(op.native_len, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    rc = L.fg_op_apply_native_noalloc(op.handle, x.data_ptr(), y.data_ptr(), 0, 0)
    assert rc == femgpu.FG_INVALID_ARGUMENT
    assert "static scratch array" in femgpu.last_error()
    op.close()
