"""femgpu -- Python front end of libfemgpu.so (the sm_100a PA operator + PCG).

Mirrors the fem-rs operator / solver surface on top of the C ABI in
include/femgpu.h:

  * ``PADiffusionOperator`` / ``PAMassOperator`` / ``PAMassDiffusionOperator``
    with ``apply`` (y += A x), ``apply_zero`` (y = A x) and ``n_dofs``
    (crates/assembly/src/partial.rs:45-57, 65-208);
  * ``SolverConfig`` / ``SolveResult`` / ``SolverError`` and its variants
    (crates/solver/src/lib.rs:46-142);
  * ``solve_cg_operator``, ``solve_pcg_jacobi`` and ``solve_pcg_chebyshev``
    (crates/solver/src/lib.rs:198-297, crates/parallel/src/par_solver.rs:262-342).

There is no CPU fallback: importing works anywhere the shared library exists,
and every numeric call runs on the GPU or raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libfemgpu.so")

FG_OK, FG_CONVERGENCE_FAILED, FG_DIMENSION_MISMATCH, FG_BREAKDOWN = 0, 1, 2, 3
FG_UNSUPPORTED, FG_DEVICE_TIMEOUT, FG_BOUNDS, FG_CUDA_ERROR, FG_INVALID_ARGUMENT = 4, 5, 6, 7, 8
MASS, DIFF, MASS_DIFF = 1, 2, 3
HOST, DEVICE = 0, 1
PC_NONE, PC_JACOBI, PC_CHEBYSHEV, PC_CHEB_NN = 0, 1, 2, 3
FP64, FP32_IR = 0, 1
QDATA_FULL, QDATA_AFFINE = 0, 1
TAG_ALL = 63

# every symbol include/femgpu.h declares
EXPORTS = ("fg_cfg_default", "fg_last_error", "fg_op_create", "fg_op_destroy", "fg_op_ndofs",
           "fg_op_layout", "fg_op_native_len", "fg_op_set_stream", "fg_op_apply",
           "fg_op_apply_native", "fg_op_diagonal", "fg_pcg", "fg_op_check",
           "fg_op_apply_native_noalloc", "fg_op_apply_f32", "fg_op_apply_native_f32",
           "fg_op_set_qdata_format", "fg_sdirk2", "fg_batch_pcg",
           "fg_unet_create", "fg_unet_destroy", "fg_unet_num_params", "fg_unet_get_params",
           "fg_unet_set_params", "fg_unet_get_grads", "fg_unet_forward", "fg_unet_loss_grad",
           "fg_unet_train_step", "fg_op_set_nodal_kappa", "fg_op_attach_unet", "fg_op_collect_pairs",
           "fg_op_collect_residuals", "fg_unet_train_energy", "fg_quadrature_points",
           "fg_assemble_source", "fg_l2_error", "fg_lumped_mass", "fg_lumped_apply", "fg_op_set_tile",
           "fg_op_tile", "fg_batch_autotune", "fg_tet_create", "fg_tet_destroy", "fg_tet_ndofs", "fg_tet_nq",
           "fg_tet_quadrature_points", "fg_tet_apply", "fg_tet_diagonal", "fg_op_set_wait_limit",
           "fg_op_create_hex", "fg_op_chunks", "fg_vec_dots", "fg_vec_pcg_update", "fg_vec_pupdate",
           "fg_tet_apply_native", "fg_tet_set_stream", "fg_tet_check")


class FgMesh(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("vcoord", C.c_void_p)]


class FgCfg(C.Structure):
    _fields_ = [("rtol", C.c_double), ("atol", C.c_double), ("max_iter", C.c_int32),
                ("print_level", C.c_int32), ("precond", C.c_int32), ("cheb_degree", C.c_int32),
                ("precision", C.c_int32), ("power_iters", C.c_int32), ("lmax", C.c_double),
                ("lmin_ratio", C.c_double), ("lmax_safety", C.c_double), ("inner_rtol", C.c_double),
                ("check_interval", C.c_int32), ("nn_budget", C.c_int32), ("nn_iter_ratio", C.c_double)]


class FgSdirkResult(C.Structure):
    _fields_ = [("steps", C.c_int32), ("max_stage_iterations", C.c_int32), ("total_iterations", C.c_int64),
                ("failed_solves", C.c_int32), ("reserved", C.c_int32), ("applies", C.c_int64),
                ("time_ms", C.c_double)]


TUNE_TZ = (1, 2, 4, 8, 16)


class FgTuneEntry(C.Structure):
    _fields_ = [("order", C.c_int32), ("kind", C.c_int32), ("format", C.c_int32), ("size_class", C.c_int32),
                ("instances", C.c_int32), ("tz", C.c_int32), ("us", C.c_double * len(TUNE_TZ)),
                ("us_other", C.c_double * len(TUNE_TZ))]


class FgResult(C.Structure):
    _fields_ = [("converged", C.c_int32), ("iterations", C.c_int32), ("final_residual", C.c_double),
                ("true_residual", C.c_double), ("status", C.c_int32), ("outer_iterations", C.c_int32),
                ("applies", C.c_int64), ("lmax", C.c_double), ("solve_ms", C.c_double),
                ("nn_fallback", C.c_int32), ("reserved", C.c_int32)]


_lib = None


def lib():
    """Load libfemgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libfemgpu.so not built ({LIB_PATH}); run `make -C fem-rs_b200`")
        L = C.CDLL(LIB_PATH)
        vp, i, d, i64 = C.c_void_p, C.c_int, C.c_double, C.c_int64
        L.fg_cfg_default.argtypes = [vp]
        L.fg_last_error.argtypes = [C.c_char_p, C.c_size_t]
        L.fg_op_create.argtypes = [vp, i, i, i, d, d, vp, d, vp, d, i, C.POINTER(vp)]
        L.fg_op_destroy.argtypes = [vp]
        L.fg_op_destroy.restype = None
        L.fg_op_ndofs.argtypes = [vp]
        L.fg_op_ndofs.restype = i64
        L.fg_op_native_len.argtypes = [vp]
        L.fg_op_native_len.restype = i64
        L.fg_op_layout.argtypes = [vp, vp]
        L.fg_op_set_stream.argtypes = [vp, vp]
        L.fg_op_apply.argtypes = [vp, vp, vp, i, i, i]
        L.fg_op_apply_native.argtypes = [vp, vp, vp, i, i]
        L.fg_op_diagonal.argtypes = [vp, vp, i, i]
        L.fg_pcg.argtypes = [vp, vp, vp, vp, vp, i]
        L.fg_op_check.argtypes = [vp]
        L.fg_op_apply_f32.argtypes = [vp, vp, vp, i, i, i]
        L.fg_op_set_qdata_format.argtypes = [vp, i]
        L.fg_sdirk2.argtypes = [vp, vp, vp, d, i, vp, vp, i]
        L.fg_batch_pcg.argtypes = [vp, i, vp, vp, vp, vp, i]
        L.fg_unet_create.argtypes = [vp, C.c_uint64, C.POINTER(vp)]
        L.fg_unet_destroy.argtypes = [vp]
        L.fg_unet_destroy.restype = None
        L.fg_unet_num_params.argtypes = [vp]
        L.fg_unet_num_params.restype = i64
        for nm in ("fg_unet_get_params", "fg_unet_set_params", "fg_unet_get_grads"):
            getattr(L, nm).argtypes = [vp, vp]
        L.fg_unet_forward.argtypes = [vp, vp, i, i, i, i, vp, i]
        L.fg_unet_loss_grad.argtypes = [vp, vp, vp, i, i, i, i, vp, i]
        L.fg_unet_train_step.argtypes = [vp, vp, vp, i, i, i, i, C.c_float, vp, i]
        L.fg_op_set_nodal_kappa.argtypes = [vp, vp, i]
        L.fg_op_attach_unet.argtypes = [vp, vp]
        L.fg_op_collect_pairs.argtypes = [vp, vp, vp, i, i, vp, vp, vp]
        L.fg_op_collect_residuals.argtypes = [vp, vp, vp, i, i, vp, vp]
        L.fg_unet_train_energy.argtypes = [vp, vp, vp, i, C.c_float, vp]
        L.fg_quadrature_points.argtypes = [vp, i, vp, i]
        L.fg_assemble_source.argtypes = [vp, i, vp, d, i, vp, i]
        L.fg_l2_error.argtypes = [vp, i, i, vp, vp, vp, i]
        L.fg_lumped_mass.argtypes = [vp, i, vp, d, vp, i]
        L.fg_lumped_apply.argtypes = [vp, vp, vp, i64, i, i]
        L.fg_op_set_tile.argtypes = [vp, i]
        L.fg_op_tile.argtypes = [vp, vp]
        L.fg_batch_autotune.argtypes = [vp, i, i, vp, i, vp]
        L.fg_tet_create.argtypes = [i, i64, vp, i64, vp, i64, i, d, d, vp, d, vp, d, i, vp, C.POINTER(vp)]
        L.fg_tet_destroy.argtypes = [vp]
        L.fg_tet_destroy.restype = None
        L.fg_tet_ndofs.argtypes = [vp]
        L.fg_tet_ndofs.restype = i64
        L.fg_tet_nq.argtypes = [vp]
        L.fg_tet_quadrature_points.argtypes = [vp, vp, i]
        L.fg_tet_apply.argtypes = [vp, vp, vp, i, i, i]
        L.fg_tet_diagonal.argtypes = [vp, vp, i, i]
        L.fg_op_apply_native_f32.argtypes = [vp, vp, vp, i, i]
        L.fg_op_set_wait_limit.argtypes = [vp, d]
        L.fg_op_create_hex.argtypes = [i, i64, vp, i64, vp, vp, i64, i, d, d, vp, d, vp, d, vp, i64,
                                       C.POINTER(vp)]
        L.fg_op_chunks.argtypes = [vp]
        L.fg_op_chunks.restype = i64
        L.fg_vec_dots.argtypes = [vp, i64, i, vp, vp, vp]
        L.fg_vec_pcg_update.argtypes = [vp, i64, vp, vp, vp, vp, vp, vp, vp, vp]
        L.fg_vec_pupdate.argtypes = [vp, vp, vp, vp, vp]
        L.fg_tet_apply_native.argtypes = [vp, vp, vp, i, i]
        L.fg_tet_set_stream.argtypes = [vp, vp]
        L.fg_tet_check.argtypes = [vp]
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(512)
    lib().fg_last_error(buf, 512)
    return buf.value.decode()


# --------------------------------------------------------------------------
# errors (crates/solver/src/lib.rs:46-54)
# --------------------------------------------------------------------------
class SolverError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


class ConvergenceFailed(SolverError):
    pass


class DimensionMismatch(SolverError):
    pass


class Breakdown(SolverError):
    """SolverError::Linger("CG operator breakdown: p^T A p is near zero")."""


class DeviceError(SolverError):
    pass


def _check(rc):
    if rc == FG_OK:
        return
    msg = last_error()
    cls = {FG_CONVERGENCE_FAILED: ConvergenceFailed, FG_DIMENSION_MISMATCH: DimensionMismatch,
           FG_BREAKDOWN: Breakdown}.get(rc, DeviceError)
    raise cls(rc, f"femgpu status {rc}: {msg}")


# --------------------------------------------------------------------------
# config / result (crates/solver/src/lib.rs:70-142)
# --------------------------------------------------------------------------
@dataclass
class SolverConfig:
    rtol: float = 1e-8
    atol: float = 0.0
    max_iter: int = 1000
    verbose: bool = False
    print_level: int = 0
    cheb_degree: int = 4
    power_iters: int = 20
    lmax: float = 0.0
    lmin_ratio: float = 30.0
    lmax_safety: float = 1.1
    precision: int = FP64
    inner_rtol: float = 0.1
    check_interval: int = 10
    nn_budget: int = 0
    nn_iter_ratio: float = 0.0

    def to_c(self, precond):
        c = FgCfg()
        lib().fg_cfg_default(C.byref(c))
        c.rtol, c.atol, c.max_iter = self.rtol, self.atol, self.max_iter
        c.print_level = self.print_level or (2 if self.verbose else 0)
        c.precond, c.cheb_degree, c.precision = precond, self.cheb_degree, self.precision
        c.power_iters, c.lmax, c.lmin_ratio = self.power_iters, self.lmax, self.lmin_ratio
        c.lmax_safety, c.inner_rtol, c.check_interval = self.lmax_safety, self.inner_rtol, self.check_interval
        c.nn_budget, c.nn_iter_ratio = self.nn_budget, self.nn_iter_ratio
        return c


@dataclass
class SolveResult:
    converged: bool
    iterations: int
    final_residual: float
    true_residual: float = 0.0
    applies: int = 0
    lmax: float = 0.0
    solve_ms: float = 0.0
    outer_iterations: int = 1
    status: int = 0
    extra: dict = field(default_factory=dict)


# --------------------------------------------------------------------------
# operators
# --------------------------------------------------------------------------
def _as_f64(a):
    """(pointer, mem, keepalive) for a numpy array or a CUDA torch tensor."""
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise TypeError("expected a C-contiguous float64 array")
        return a.ctypes.data, HOST
    mod = type(a).__module__
    if mod.startswith("torch"):
        if a.dtype.__repr__() != "torch.float64" or not a.is_contiguous():
            raise TypeError("expected a contiguous float64 tensor")
        return a.data_ptr(), (DEVICE if a.is_cuda else HOST)
    raise TypeError(f"unsupported array type {type(a)}")


class PAOperator:
    """Matrix-free PA operator on a structured hex box (sm_100a kernels).

    ``mesh``: (nx, ny, nz) or dict(nx=, ny=, nz=, vcoord=array((nx+1)(ny+1)(nz+1), 3)).
    ``kappa`` / ``rho``: scalar or per-quadrature-point array [E][qz][qy][qx].
    ``ess_tags``: Dirichlet boundary tags (bit t-1 = tag t) for the constrained form.
    """

    def __init__(self, mesh, order, kind=DIFF, kappa=1.0, rho=1.0, c_mass=1.0, c_diff=1.0,
                 ess_tags=TAG_ALL, quad_order=None):
        if isinstance(mesh, dict):
            nx, ny, nz, vc = mesh["nx"], mesh["ny"], mesh["nz"], mesh.get("vcoord")
        else:
            (nx, ny, nz), vc = mesh, None
        self.nx, self.ny, self.nz, self.order, self.kind = int(nx), int(ny), int(nz), int(order), kind
        nq = order + 1 if quad_order is None else (int(quad_order) + 2) // 2
        self._vc = None if vc is None else np.ascontiguousarray(vc, dtype=np.float64)
        m = FgMesh(self.nx, self.ny, self.nz, None if self._vc is None else self._vc.ctypes.data)
        kq = None if np.isscalar(kappa) else np.ascontiguousarray(kappa, dtype=np.float64)
        rq = None if np.isscalar(rho) else np.ascontiguousarray(rho, dtype=np.float64)
        E = self.nx * self.ny * self.nz
        for arr in (kq, rq):
            if arr is not None and arr.size != E * nq ** 3:
                raise DimensionMismatch(FG_DIMENSION_MISMATCH, "coefficient array has wrong size")
        h = C.c_void_p()
        rc = lib().fg_op_create(C.byref(m), self.order, nq, kind, float(c_mass), float(c_diff),
                                None if kq is None else kq.ctypes.data,
                                float(kappa) if kq is None else 0.0,
                                None if rq is None else rq.ctypes.data,
                                float(rho) if rq is None else 0.0, int(ess_tags), C.byref(h))
        _check(rc)
        self._h = h
        dims = (C.c_int64 * 4)()
        lib().fg_op_layout(self._h, dims)
        self.NI, self.NJ, self.NK, self.NIp = (int(v) for v in dims)

    def close(self):
        if getattr(self, "_h", None):
            lib().fg_op_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # MatFreeOperator
    def n_dofs(self):
        return int(lib().fg_op_ndofs(self._h))

    @property
    def native_len(self):
        return int(lib().fg_op_native_len(self._h))

    def _apply(self, x, y, accumulate, constrained):
        n = self.n_dofs()
        if len(x) != n or len(y) != n:
            raise DimensionMismatch(FG_DIMENSION_MISMATCH, f"operator is {n}x{n}, vectors {len(x)}/{len(y)}")
        px, mx = _as_f64(x)
        py, my = _as_f64(y)
        if mx != my:
            raise TypeError("x and y must live in the same memory space")
        _check(lib().fg_op_apply(self._h, px, py, int(accumulate), int(constrained), mx))
        return y

    def apply(self, x, y, constrained=False):
        """y += A x (does not zero y first), partial.rs:46-47."""
        return self._apply(x, y, True, constrained)

    def apply_zero(self, x, y, constrained=False):
        """y = A x, partial.rs:50-53."""
        return self._apply(x, y, False, constrained)

    def matvec(self, x, constrained=False):
        y = np.zeros(self.n_dofs())
        return self.apply_zero(np.ascontiguousarray(x, dtype=np.float64), y, constrained)

    def apply_native(self, x_ptr, y_ptr, accumulate=False, constrained=True):
        """Device pointers in the native (padded) layout; asynchronous."""
        _check(lib().fg_op_apply_native(self._h, x_ptr, y_ptr, int(accumulate), int(constrained)))

    def apply_native_f32(self, x_ptr, y_ptr, accumulate=False, constrained=True):
        """FP32 apply on float32 device vectors in the native layout; asynchronous."""
        _check(lib().fg_op_apply_native_f32(self._h, x_ptr, y_ptr, int(accumulate), int(constrained)))

    def set_qdata_format(self, fmt):
        """QDATA_FULL (general geometry) or QDATA_AFFINE (constant-J elements only)."""
        _check(lib().fg_op_set_qdata_format(self._h, int(fmt)))

    def diagonal(self, constrained=True):
        d = np.zeros(self.n_dofs())
        _check(lib().fg_op_diagonal(self._h, d.ctypes.data, int(constrained), HOST))
        return d

    def check(self):
        _check(lib().fg_op_check(self._h))

    def set_wait_limit(self, seconds):
        """Limit of each device-side wait of the apply kernels (<= 0: the 1 s default)."""
        _check(lib().fg_op_set_wait_limit(self._h, C.c_double(seconds)))

    def set_stream(self, stream_ptr):
        _check(lib().fg_op_set_stream(self._h, stream_ptr))

    @property
    def tile(self):
        """(32, WY, TZ): elements per apply work item in x, y, z."""
        d = (C.c_int * 3)()
        _check(lib().fg_op_tile(self._h, d))
        return tuple(d)

    def set_tile(self, tz):
        """Re-lay out the quadrature data for items of TZ = tz element layers."""
        _check(lib().fg_op_set_tile(self._h, int(tz)))

    # native layout helpers
    def to_native(self, v):
        out = np.zeros((self.NK, self.NJ, self.NIp))
        out[:, :, :self.NI] = np.asarray(v).reshape(self.NK, self.NJ, self.NI)
        return out.ravel()

    def from_native(self, v):
        return np.asarray(v).reshape(self.NK, self.NJ, self.NIp)[:, :, :self.NI].ravel()

    # solver
    def pcg(self, b, x, cfg: SolverConfig, precond) -> SolveResult:
        n = self.n_dofs()
        if len(b) != n or len(x) != n:
            raise DimensionMismatch(FG_DIMENSION_MISMATCH, f"matrix is {n}x{n}, rhs has length {len(b)}")
        pb, mb = _as_f64(b)
        px, mx = _as_f64(x)
        if mb != mx:
            raise TypeError("b and x must live in the same memory space")
        c = cfg.to_c(precond)
        r = FgResult()
        rc = lib().fg_pcg(self._h, pb, px, C.byref(c), C.byref(r), mb)
        res = SolveResult(bool(r.converged), int(r.iterations), float(r.final_residual),
                          float(r.true_residual), int(r.applies), float(r.lmax), float(r.solve_ms),
                          int(r.outer_iterations), int(r.status), extra={"nn_fallback": int(r.nn_fallback)})
        if rc not in (FG_OK, FG_CONVERGENCE_FAILED):
            _check(rc)
        return res


class HexMeshOperator(PAOperator):
    """PA operator on an unstructured Hex8 mesh: PAMassOperator /
    PADiffusionOperator::new over any connectivity and DOF numbering
    (partial.rs:65-80, 138-149 with the Hex8 geometry of assembler.rs:96-143).

    ``coords``: (n_nodes, 3); ``conn``: (E, 8) vertex ids in HexQ1 order
    (hex.rs:27-36); ``elem_dofs``: (E, (p+1)^3) element DOF maps (order 1: None
    means DOF = node, as DofManager::build_p1; orders 2-3: tensor order on the
    reference cube, local DOF (c, b, a) at (c*(p+1) + b)*(p+1) + a);
    ``kappa`` / ``rho``: scalar or (E, (p+1)^3) at the tensor Gauss points;
    ``ess_dofs``: the essential-DOF list (boundary_dofs, constraints.rs:53-60).
    Native vectors are the plain numbering padded with zeros to a multiple of 4.  The scatter works on
    Morton-ordered element chunks with the DOF sums in shared memory (no float atomics, same sums every
    run).
    """

    def __init__(self, order, coords, conn, elem_dofs=None, n_dofs=None, kind=DIFF, kappa=1.0, rho=1.0,
                 c_mass=1.0, c_diff=1.0, ess_dofs=None):
        self.order, self.kind = int(order), kind
        xyz = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
        cn = np.ascontiguousarray(conn, dtype=np.uint32).reshape(-1, 8)
        E = cn.shape[0]
        nl = (self.order + 1) ** 3
        ed = None if elem_dofs is None else np.ascontiguousarray(elem_dofs, dtype=np.uint32).reshape(E, nl)
        if n_dofs is None:
            n_dofs = xyz.shape[0] if ed is None else int(ed.max()) + 1
        kq = None if np.isscalar(kappa) else np.ascontiguousarray(kappa, dtype=np.float64)
        rq = None if np.isscalar(rho) else np.ascontiguousarray(rho, dtype=np.float64)
        for arr in (kq, rq):
            if arr is not None and arr.size != E * nl:
                raise DimensionMismatch(FG_DIMENSION_MISMATCH, "coefficient array has wrong size")
        ess = None if ess_dofs is None else np.ascontiguousarray(ess_dofs, dtype=np.uint32)
        h = C.c_void_p()
        rc = lib().fg_op_create_hex(self.order, xyz.shape[0], xyz.ctypes.data, E, cn.ctypes.data,
                                    None if ed is None else ed.ctypes.data, int(n_dofs), kind, float(c_mass),
                                    float(c_diff), None if kq is None else kq.ctypes.data,
                                    float(kappa) if kq is None else 0.0, None if rq is None else rq.ctypes.data,
                                    float(rho) if rq is None else 0.0, None if ess is None else ess.ctypes.data,
                                    0 if ess is None else ess.size, C.byref(h))
        _check(rc)
        self._h = h
        self.nx = self.ny = self.nz = None
        dims = (C.c_int64 * 4)()
        lib().fg_op_layout(self._h, dims)
        self.NI, self.NJ, self.NK, self.NIp = (int(v) for v in dims)

    @property
    def chunks(self):
        """Element chunks of the deterministic scatter (one CTA each)."""
        return int(lib().fg_op_chunks(self._h))


class PADiffusionOperator(PAOperator):
    """PADiffusionOperator::new(space, kappa, quad_order) (partial.rs:138-149)."""

    def __init__(self, mesh, order, kappa=1.0, quad_order=None, ess_tags=TAG_ALL):
        super().__init__(mesh, order, DIFF, kappa=kappa, quad_order=quad_order, ess_tags=ess_tags)


class PAMassOperator(PAOperator):
    """PAMassOperator::new(space, rho, quad_order) (partial.rs:65-80)."""

    def __init__(self, mesh, order, rho=1.0, quad_order=None, ess_tags=TAG_ALL):
        super().__init__(mesh, order, MASS, rho=rho, quad_order=quad_order, ess_tags=ess_tags)


class PAMassDiffusionOperator(PAOperator):
    """c_mass M + c_diff K in one apply (the SDIRK stage matrix M + gamma dt K of
    examples/mfem_ex10_heat_equation.rs:141-156, matrix-free)."""

    def __init__(self, mesh, order, c_mass, c_diff, kappa=1.0, rho=1.0, ess_tags=TAG_ALL):
        super().__init__(mesh, order, MASS_DIFF, kappa=kappa, rho=rho, c_mass=c_mass,
                         c_diff=c_diff, ess_tags=ess_tags)


# --------------------------------------------------------------------------
# solver entry points
# --------------------------------------------------------------------------
def _finish(res: SolveResult, cfg: SolverConfig, raise_on_fail: bool):
    if raise_on_fail and not res.converged:
        if res.status == FG_BREAKDOWN:
            raise Breakdown(FG_BREAKDOWN, "CG operator breakdown: p^T A p is near zero")
        raise ConvergenceFailed(FG_CONVERGENCE_FAILED,
                                f"solver did not converge in {cfg.max_iter} iterations "
                                f"(residual = {res.final_residual:.3e})")
    return res


def solve_cg_operator(nrows, ncols, op: PAOperator, b, x, cfg=None):
    """Unpreconditioned CG over the constrained operator (lib.rs:198-278);
    raises ConvergenceFailed / Breakdown like the reference's Err variants."""
    cfg = cfg or SolverConfig()
    if nrows != ncols or len(b) != nrows or len(x) != ncols or op.n_dofs() != nrows:
        raise DimensionMismatch(FG_DIMENSION_MISMATCH,
                                f"dimension mismatch: matrix is {nrows}x{ncols}, rhs has length {len(b)}")
    return _finish(op.pcg(b, x, cfg, PC_NONE), cfg, True)


def solve_pcg_jacobi(op: PAOperator, b, x, cfg=None):
    """PCG + Jacobi (lib.rs:281-297, par_solver.rs:262-342): returns a
    SolveResult with converged=False instead of raising on non-convergence."""
    cfg = cfg or SolverConfig()
    return op.pcg(b, x, cfg, PC_JACOBI)


def solve_pcg_chebyshev(op: PAOperator, b, x, cfg=None):
    """PCG with a Chebyshev(D^-1 A) preconditioner of cfg.cheb_degree sweeps."""
    cfg = cfg or SolverConfig()
    return op.pcg(b, x, cfg, PC_CHEBYSHEV)


def batch_pcg(ops, bs, xs, cfg=None, precond=PC_CHEBYSHEV):
    """Solve n independent systems together (fg_batch_pcg): FP32 mixed-precision
    PCG, one launch per phase over all instances, CUDA-graph replayed.  Returns
    (all_converged, [SolveResult])."""
    cfg = cfg or SolverConfig(rtol=1e-8, precision=FP32_IR)
    n = len(ops)
    hs = (C.c_void_p * n)(*[o.handle for o in ops])
    pb = (C.c_void_p * n)()
    px = (C.c_void_p * n)()
    mem = None
    for i in range(n):
        pb[i], m1 = _as_f64(bs[i])
        px[i], m2 = _as_f64(xs[i])
        mem = m1 if mem is None else mem
        if m1 != mem or m2 != mem:
            raise TypeError("all vectors must live in one memory space")
    res = (FgResult * n)()
    c = cfg.to_c(precond)
    rc = lib().fg_batch_pcg(hs, n, pb, px, C.byref(c), res, mem)
    if rc not in (FG_OK, FG_CONVERGENCE_FAILED):
        _check(rc)
    out = [SolveResult(bool(r.converged), int(r.iterations), float(r.final_residual), float(r.true_residual),
                       int(r.applies), float(r.lmax), float(r.solve_ms), int(r.outer_iterations), int(r.status))
           for r in res]
    return rc == FG_OK, out


def batch_autotune(ops, reps=5):
    """Choose each batch class's quadrature-data format and item depth TZ by
    timing the batched FP32 apply (fg_batch_autotune); the choice stays on the
    operators.  Returns one dict per (order, kind, size class): ``format`` and
    ``tz`` chosen, ``us`` the times per TZ in that format, ``us_other`` in the
    other format (None: not tried)."""
    n = len(ops)
    hs = (C.c_void_p * n)(*[o.handle for o in ops])
    out = (FgTuneEntry * 64)()
    cnt = C.c_int()
    _check(lib().fg_batch_autotune(hs, n, int(reps), out, 64, C.byref(cnt)))
    return [dict(order=e.order, kind=e.kind, format=e.format, size_class=e.size_class, instances=e.instances,
                 tz=e.tz, us={tz: (e.us[k] if e.us[k] >= 0 else None) for k, tz in enumerate(TUNE_TZ)},
                 us_other={tz: (e.us_other[k] if e.us_other[k] >= 0 else None) for k, tz in enumerate(TUNE_TZ)})
            for e in out[:min(cnt.value, 64)]]


SDIRK2_GAMMA = 1.0 - 2.0 ** -0.5  # crates/solver/src/ode.rs:441


def sdirk2(stiff: PAOperator, stage: PAOperator, u, dt, n_steps, cfg=None, precond=PC_JACOBI):
    """SDIRK-2 heat stepping (examples/mfem_ex10_heat_equation.rs:201-250) on the
    device; ``stage`` must be M + gamma*dt*K.  ``u`` is updated in place.
    Returns a dict with iteration counts and the device time."""
    cfg = cfg or SolverConfig(rtol=1e-10)
    pu, mu = _as_f64(u)
    r = FgSdirkResult()
    rc = lib().fg_sdirk2(stiff.handle, stage.handle, pu, float(dt), int(n_steps),
                         C.byref(cfg.to_c(precond)), C.byref(r), mu)
    _check(rc)
    return dict(steps=r.steps, total_iterations=int(r.total_iterations),
                max_stage_iterations=r.max_stage_iterations, applies=int(r.applies), time_ms=r.time_ms)


class UNet:
    """Learned coarse correction network (fg_unet): BF16 3-D U-net, FP32
    accumulation, trained by the library's own forward/backward kernels."""

    def __init__(self, channels=(16, 32, 48), seed=0):
        self.channels = tuple(int(c) for c in channels)
        h = C.c_void_p()
        ch = (C.c_int * 3)(*self.channels)
        _check(lib().fg_unet_create(ch, int(seed), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().fg_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def num_params(self):
        return int(lib().fg_unet_num_params(self._h))

    def get_params(self):
        a = np.zeros(self.num_params, dtype=np.float32)
        _check(lib().fg_unet_get_params(self._h, a.ctypes.data))
        return a

    def set_params(self, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        assert a.size == self.num_params
        _check(lib().fg_unet_set_params(self._h, a.ctypes.data))

    def get_grads(self):
        a = np.zeros(self.num_params, dtype=np.float32)
        _check(lib().fg_unet_get_grads(self._h, a.ctypes.data))
        return a

    def forward(self, inp):
        """inp: float32 [B,Z,Y,X,2] (numpy) -> [B,Z,Y,X]"""
        inp = np.ascontiguousarray(inp, dtype=np.float32)
        B, Z, Y, X, _ = inp.shape
        out = np.zeros((B, Z, Y, X), dtype=np.float32)
        _check(lib().fg_unet_forward(self._h, inp.ctypes.data, B, Z, Y, X, out.ctypes.data, HOST))
        return out

    def _step(self, fn, inp, target, *extra):
        loss = C.c_float()
        if isinstance(inp, np.ndarray):
            inp = np.ascontiguousarray(inp, dtype=np.float32)
            target = np.ascontiguousarray(target, dtype=np.float32)
            B, Z, Y, X, _ = inp.shape
            _check(fn(self._h, inp.ctypes.data, target.ctypes.data, B, Z, Y, X, *extra, C.byref(loss), HOST))
        else:  # torch CUDA tensors
            B, Z, Y, X, _ = inp.shape
            _check(fn(self._h, inp.data_ptr(), target.data_ptr(), B, Z, Y, X, *extra, C.byref(loss), DEVICE))
        return float(loss.value)

    def loss_grad(self, inp, target):
        return self._step(lib().fg_unet_loss_grad, inp, target)

    def train_step(self, inp, target, lr):
        return self._step(lib().fg_unet_train_step, inp, target, C.c_float(lr))

    def train_energy(self, op, res, lr):
        """One Adam step on the energy loss of the residuals ``res`` (torch CUDA
        float64 tensor [B, native_len]) for the operator ``op``; returns the
        batch-mean loss (c.Ac/2 - c.r) / (s^2 Nc)."""
        assert res.dtype.is_floating_point and res.element_size() == 8 and res.is_contiguous()
        assert res.shape[-1] == op.native_len
        loss = C.c_float()
        _check(lib().fg_unet_train_energy(self._h, op.handle, res.data_ptr(), int(res.shape[0]),
                                          C.c_float(lr), C.byref(loss)))
        return float(loss.value)


def set_nodal_kappa(op, kappa_nodal, levels=1):
    """kappa at the DOFs for the log-coefficient channel; ``levels`` (1 to 4)
    coarsenings between the DOF lattice and the network volume."""
    k = np.ascontiguousarray(kappa_nodal, dtype=np.float64)
    _check(lib().fg_op_set_nodal_kappa(op.handle, k.ctypes.data, int(levels)))
    op._nn_levels = int(levels)


def nn_volume(op):
    """(Z, Y, X) of the network volume of an operator after set_nodal_kappa."""
    L = getattr(op, "_nn_levels", 1)
    z, y, x = op.NK, op.NJ, op.NI
    for _ in range(L):
        z, y, x = (z + 1) // 2, (y + 1) // 2, (x + 1) // 2
    return z, y, x


def attach_unet(op, net):
    _check(lib().fg_op_attach_unet(op.handle, None if net is None else net.handle))


def collect_pairs(op, b, every, max_pairs, cfg=None):
    """Training pairs (torch CUDA float32 tensors in [n,Zc,Yc,Xc,2], target [n,Zc,Yc,Xc])."""
    import torch
    cfg = cfg or SolverConfig(rtol=1e-10, max_iter=20000)
    Zc, Yc, Xc = nn_volume(op)
    din = torch.zeros((max_pairs, Zc, Yc, Xc, 2), dtype=torch.float32, device="cuda")
    dt = torch.zeros((max_pairs, Zc, Yc, Xc), dtype=torch.float32, device="cuda")
    b = np.ascontiguousarray(b, dtype=np.float64)
    npairs = C.c_int()
    c = cfg.to_c(PC_CHEBYSHEV)
    _check(lib().fg_op_collect_pairs(op.handle, b.ctypes.data, C.byref(c), int(every), int(max_pairs),
                                     din.data_ptr(), dt.data_ptr(), C.byref(npairs)))
    n = npairs.value
    return din[:n], dt[:n]


def collect_residuals(op, b, every, max_res, cfg=None):
    """Recurrence residuals of a plain Chebyshev-PCG solve from x0 = 0 at
    iterations 0, every, 2*every, ... (torch CUDA float64 [n, native_len])."""
    import torch
    cfg = cfg or SolverConfig(rtol=1e-10, max_iter=20000)
    out = torch.zeros((max_res, op.native_len), dtype=torch.float64, device="cuda")
    b = np.ascontiguousarray(b, dtype=np.float64)
    n = C.c_int()
    c = cfg.to_c(PC_CHEBYSHEV)
    _check(lib().fg_op_collect_residuals(op.handle, b.ctypes.data, C.byref(c), int(every), int(max_res),
                                         out.data_ptr(), C.byref(n)))
    return out[:n.value]


class TetOperator:
    """PA mass / diffusion operator on an unstructured Tet4 mesh with TetP1, TetP2
    or TetP3 (fg_tet_*): the MatFreeOperator surface of partial.rs (apply =
    y += A x, apply_zero = y = A x, n_dofs) plus the Jacobi diagonal.
    coords [n_nodes, 3]; elem_dofs [E, 4|10|20] (first 4 = vertex nodes);
    kappa / rho: constants or [E, nq] tables at quadrature_points()."""

    def __init__(self, p, coords, elem_dofs, n_dofs, kind=DIFF, kappa=1.0, rho=1.0, c_mass=1.0, c_diff=1.0,
                 quad_order=None, ess=None):
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        dofs = np.ascontiguousarray(elem_dofs, dtype=np.int32)
        self.p, self.n = int(p), int(n_dofs)
        self.quad_order = int(quad_order if quad_order is not None else 2 * p)
        kq = None if np.isscalar(kappa) else np.ascontiguousarray(kappa, dtype=np.float64)
        rq = None if np.isscalar(rho) else np.ascontiguousarray(rho, dtype=np.float64)
        ms = None if ess is None else np.ascontiguousarray(ess, dtype=np.uint8)
        self._keep = (coords, dofs, kq, rq, ms)
        h = C.c_void_p()
        _check(lib().fg_tet_create(self.p, coords.shape[0], coords.ctypes.data, dofs.shape[0], dofs.ctypes.data,
                                   self.n, int(kind), float(c_mass), float(c_diff),
                                   None if kq is None else kq.ctypes.data, float(kappa) if kq is None else 0.0,
                                   None if rq is None else rq.ctypes.data, float(rho) if rq is None else 0.0,
                                   self.quad_order, None if ms is None else ms.ctypes.data, C.byref(h)))
        self._h = h
        self.nq = int(lib().fg_tet_nq(h))

    def close(self):
        if getattr(self, "_h", None):
            lib().fg_tet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def n_dofs(self):
        return int(lib().fg_tet_ndofs(self._h))

    def quadrature_points(self):
        n_elem = self._keep[1].shape[0]
        out = np.zeros((n_elem, self.nq, 3))
        _check(lib().fg_tet_quadrature_points(self._h, out.ctypes.data, HOST))
        return out

    def _apply(self, x, y, accumulate, constrained):
        px, mx = _as_f64(x)
        py, my = _as_f64(y)
        if mx != my:
            raise TypeError("x and y must live in one memory space")
        _check(lib().fg_tet_apply(self._h, px, py, int(accumulate), int(constrained), mx))
        return y

    def apply(self, x, y, constrained=False):
        """y += A x"""
        return self._apply(x, y, True, constrained)

    def apply_zero(self, x, y, constrained=False):
        """y = A x"""
        return self._apply(x, y, False, constrained)

    def matvec(self, x, constrained=False):
        y = np.zeros(self.n)
        return self.apply_zero(np.ascontiguousarray(x, dtype=np.float64), y, constrained)

    def diagonal(self, constrained=False):
        d = np.zeros(self.n)
        _check(lib().fg_tet_diagonal(self._h, d.ctypes.data, int(constrained), HOST))
        return d

    def apply_native(self, x_ptr, y_ptr, accumulate=False, constrained=True):
        """y (+)= A x on device pointers, asynchronous on the handle's stream."""
        _check(lib().fg_tet_apply_native(self._h, x_ptr, y_ptr, int(accumulate), int(constrained)))

    def set_stream(self, stream_ptr):
        _check(lib().fg_tet_set_stream(self._h, stream_ptr))

    def check(self):
        _check(lib().fg_tet_check(self._h))


def _mesh_struct(nx, ny, nz, vcoord):
    vc = None if vcoord is None else np.ascontiguousarray(vcoord, dtype=np.float64)
    m = FgMesh(int(nx), int(ny), int(nz), None if vc is None else vc.ctypes.data)
    return m, vc


def quadrature_points(nx, ny, nz, nq, vcoord=None):
    """Physical Gauss points (nq per direction): [E, nq^3, 3]."""
    m, _vc = _mesh_struct(nx, ny, nz, vcoord)
    out = np.zeros((nx * ny * nz, nq ** 3, 3))
    _check(lib().fg_quadrature_points(C.byref(m), int(nq), out.ctypes.data, HOST))
    return out


def assemble_source(nx, ny, nz, p, f_q=None, f=1.0, ess_tags=TAG_ALL, vcoord=None):
    """b_i = sum_e sum_q w |det J| f(x_q) phi_i(x_q) (DomainSourceIntegrator +
    assemble_linear), essential rows zeroed; f_q at quadrature_points(.., p+1)."""
    m, _vc = _mesh_struct(nx, ny, nz, vcoord)
    fq = None if f_q is None else np.ascontiguousarray(f_q, dtype=np.float64)
    b = np.zeros((nx * p + 1) * (ny * p + 1) * (nz * p + 1))
    _check(lib().fg_assemble_source(C.byref(m), int(p), None if fq is None else fq.ctypes.data, float(f),
                                    int(ess_tags), b.ctypes.data, HOST))
    return b


def l2_error(nx, ny, nz, p, u, u_q=None, nq=None, vcoord=None):
    """||u_h - u||_L2 with an nq-point Gauss rule per direction (default p+2
    clamped to 4, as hex_rule does); u_q = exact values at the points of that
    rule ([E, nq^3]) or None."""
    nq = int(nq if nq is not None else min(p + 2, 4))
    m, _vc = _mesh_struct(nx, ny, nz, vcoord)
    uu = np.ascontiguousarray(u, dtype=np.float64)
    uq = None if u_q is None else np.ascontiguousarray(u_q, dtype=np.float64)
    err = C.c_double()
    _check(lib().fg_l2_error(C.byref(m), int(p), nq, uu.ctypes.data, None if uq is None else uq.ctypes.data,
                             C.byref(err), HOST))
    return float(err.value)


class LumpedMassOperator:
    """LumpedMassOperator (crates/assembly/src/partial.rs:217-274): row-sum
    lumped mass diagonal assembled on the GPU; apply / apply_zero /
    apply_inverse run on the GPU."""

    def __init__(self, nx, ny, nz, p, rho=1.0, rho_q=None, vcoord=None):
        m, _vc = _mesh_struct(nx, ny, nz, vcoord)
        rq = None if rho_q is None else np.ascontiguousarray(rho_q, dtype=np.float64)
        self.diag = np.zeros((nx * p + 1) * (ny * p + 1) * (nz * p + 1))
        _check(lib().fg_lumped_mass(C.byref(m), int(p), None if rq is None else rq.ctypes.data, float(rho),
                                    self.diag.ctypes.data, HOST))

    def _run(self, x, y, mode):
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert y.dtype == np.float64 and y.flags.c_contiguous and len(x) == len(y) == len(self.diag)
        _check(lib().fg_lumped_apply(self.diag.ctypes.data, x.ctypes.data, y.ctypes.data, len(x), mode, HOST))

    def apply(self, x, y):
        """y += diag * x"""
        self._run(x, y, 1)

    def apply_zero(self, x, y):
        """y = diag * x"""
        self._run(x, y, 0)

    def apply_inverse(self, x, y):
        """y = x / diag (0 where |diag| <= 1e-14)"""
        self._run(x, y, 2)


def nodal_kappa_from_q(kq, nx, ny, nz, p=1):
    """kappa on the DOF lattice ((p*nz+1, p*ny+1, p*nx+1), plain layout): at each
    lattice node the mean over the elements whose closed box holds it of the
    element's mean quadrature-point kappa."""
    nq = p + 1
    try:
        import torch
        if isinstance(kq, torch.Tensor):
            kq = kq.detach().double().cpu().numpy()
    except ImportError:
        pass
    k = np.asarray(kq, dtype=np.float64).reshape(nz, ny, nx, nq ** 3).mean(axis=-1)
    acc = np.zeros((p * nz + 1, p * ny + 1, p * nx + 1))
    cnt = np.zeros_like(acc)
    for dz in range(p + 1):
        for dy in range(p + 1):
            for dx in range(p + 1):
                sl = (slice(dz, dz + p * nz, p), slice(dy, dy + p * ny, p), slice(dx, dx + p * nx, p))
                acc[sl] += k
                cnt[sl] += 1
    return (acc / cnt).ravel()


def unit_cube_vertices(nx, ny, nz):
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    return np.stack([i / nx, j / ny, k / nz], axis=-1).reshape(-1, 3).astype(np.float64)
