"""Sharded PA operator and Jacobi-PCG over a z-slab element partition.

One rank per GPU.  The distributed form of the reference's solve path
(crates/parallel):

  * element partition: each rank owns a contiguous range of element layers
    in z, the box form of the element ownership of partition.rs; the rank's
    local problem is a PA operator on its slab of the structured hex mesh
    (its vertex planes and its elements' quadrature-point coefficients);
  * halo sum: after the local E^T, the DOF plane shared by ranks r and r+1
    holds a partial sum on each side.  The reference adds ghost
    contributions into the owner (GhostExchange::reverse, ghost.rs:232-262)
    and sends the owner's values back (GhostExchange::forward,
    ghost.rs:170-230).  Here both sides exchange their partial planes once
    and add the other's: a + b == b + a exactly, so both copies end
    bit-identical and every vector stays consistent without a second
    exchange;
  * ParVector::global_dot (par_vector.rs:182-194): the local dot over owned
    DOFs, then CommBackend::allreduce_sum_f64 (backend/mod.rs:56);
  * par_solve_pcg_jacobi (par_solver.rs:262-342).

DOF ownership: rank r owns its local DOF planes 0 .. NK-2; its top plane is
owned by rank r+1 (whose plane 0 it is), except on the last rank, which owns
all of its planes.  Essential DOFs: the x/y boundary tags apply on every
rank, the z0 tag only on the first rank and the z1 tag only on the last;
on an interface plane the essential rows are the identity on both sides
and are not summed.

Local work runs through the C ABI on torch's current CUDA stream, with
vectors in the native padded layout of fg_op_layout: the apply, the
diagonal, and in the PCG loop the owned-DOF dots, the x / r / z update and
the direction update (fg_vec_dots, fg_vec_pcg_update, fg_vec_pupdate:
deterministic block-order sums, scalars kept on the device, one allreduce
per reduction step).  Communication goes through a ``Comm``: ``TorchComm``
(torch.distributed; NCCL between GPUs, gloo between CPU processes) or
``ThreadGroup`` ranks (threads of one process, each with its own stream).
Local operators without those entry points (the CPU oracle slabs of the
tests) take the same loop with torch tensor arithmetic.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np
import torch

from . import DEVICE, DIFF, TAG_ALL, PAOperator, SolveResult, SolverConfig, _check, lib

TAG_Z0, TAG_Z1, TAG_Y0, TAG_Y1, TAG_X0, TAG_X1 = 1, 2, 4, 8, 16, 32


def slab_partition(nz: int, world: int):
    """Contiguous element-layer ranges [z0, z1) per rank, sizes differing by
    at most one (the first nz % world ranks take one more layer)."""
    if world < 1 or nz < world:
        raise ValueError(f"cannot split {nz} element layers over {world} ranks")
    base, extra = divmod(nz, world)
    out, z = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((z, z + n))
        z += n
    return out


# ---------------------------------------------------------------------------
# communication
# ---------------------------------------------------------------------------
class Comm:
    """Interface the sharded operator needs (a subset of CommBackend,
    backend/mod.rs:40-104): rank/size, an in-place sum over ranks of a small
    float64 tensor, and the exchange of interface planes with the neighbours
    below (rank-1) and above (rank+1)."""

    rank: int = 0
    size: int = 1

    def allreduce_sum(self, t):
        raise NotImplementedError

    def exchange(self, send_lo, send_hi):
        """send_lo goes to rank-1 (None on rank 0), send_hi to rank+1 (None on
        the last rank); returns (plane from rank-1, plane from rank+1)."""
        raise NotImplementedError


class TorchComm(Comm):
    """torch.distributed process group (NCCL for CUDA tensors, gloo for CPU).
    ``rank`` / ``size`` are positions within ``group``; the neighbours of the
    plane exchange are translated to global ranks for the point-to-point
    operations, so any group works, not only the default one."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self._dist, self._group = dist, group
        self.rank, self.size = dist.get_rank(group), dist.get_world_size(group)

    def _peer(self, group_rank):
        if self._group is None:
            return group_rank
        return self._dist.get_global_rank(self._group, group_rank)

    def allreduce_sum(self, t):
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM, group=self._group)
        return t

    def exchange(self, send_lo, send_hi):
        dist = self._dist
        ops, rlo, rhi = [], None, None
        if send_lo is not None:
            rlo = torch.empty_like(send_lo)
            lo = self._peer(self.rank - 1)
            ops += [dist.P2POp(dist.isend, send_lo, lo, self._group),
                    dist.P2POp(dist.irecv, rlo, lo, self._group)]
        if send_hi is not None:
            rhi = torch.empty_like(send_hi)
            hi = self._peer(self.rank + 1)
            ops += [dist.P2POp(dist.isend, send_hi, hi, self._group),
                    dist.P2POp(dist.irecv, rhi, hi, self._group)]
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        return rlo, rhi


class ThreadGroup:
    """Ranks as threads of one process (one GPU, or CPU tensors): shared
    slots and a barrier with a timeout, so a rank that fails or never
    arrives breaks the barrier for the others instead of hanging them.
    Sums are taken in rank order on every rank (identical results)."""

    def __init__(self, size: int, timeout: float = 120.0):
        self.size = int(size)
        self.barrier = threading.Barrier(self.size, timeout=timeout)
        self.slots = [None] * self.size
        self.lo = [None] * self.size
        self.hi = [None] * self.size

    def comm(self, rank: int) -> "ThreadComm":
        return ThreadComm(self, rank)


class ThreadComm(Comm):
    def __init__(self, group: ThreadGroup, rank: int):
        self.g, self.rank, self.size = group, int(rank), group.size

    @staticmethod
    def _sync(t):
        if t is not None and t.is_cuda:
            torch.cuda.current_stream(t.device).synchronize()

    def allreduce_sum(self, t):
        g = self.g
        self._sync(t)
        g.slots[self.rank] = t
        g.barrier.wait()
        total = g.slots[0].clone()
        for i in range(1, self.size):
            total += g.slots[i]
        self._sync(total)
        g.barrier.wait()
        t.copy_(total)
        return t

    def exchange(self, send_lo, send_hi):
        g = self.g
        self._sync(send_lo)
        self._sync(send_hi)
        g.lo[self.rank], g.hi[self.rank] = send_lo, send_hi
        g.barrier.wait()
        rlo = g.hi[self.rank - 1].clone() if self.rank > 0 else None
        rhi = g.lo[self.rank + 1].clone() if self.rank < self.size - 1 else None
        self._sync(rlo)
        self._sync(rhi)
        g.barrier.wait()
        return rlo, rhi


# ---------------------------------------------------------------------------
# local operator on the rank's slab
# ---------------------------------------------------------------------------
class GpuSlab:
    """The rank's slab as a PAOperator on the current CUDA device.  Vectors
    are float64 CUDA tensors in the native layout (NK, NJ, NIp)."""

    def __init__(self, mesh, order, kind, kappa, rho, c_mass, c_diff, ess_tags):
        self.op = PAOperator(mesh, order, kind=kind, kappa=kappa, rho=rho, c_mass=c_mass, c_diff=c_diff,
                             ess_tags=ess_tags)
        self.NI, self.NJ, self.NK, self.pitch = self.op.NI, self.op.NJ, self.op.NK, self.op.NIp
        self.device = torch.device("cuda", torch.cuda.current_device())

    def _stream(self):
        self.op.set_stream(torch.cuda.current_stream(self.device).cuda_stream)

    def apply(self, x, y):
        """y = A_local x (constrained), asynchronous on the current stream."""
        self._stream()
        self.op.apply_native(x.data_ptr(), y.data_ptr(), False, True)

    def diagonal(self):
        self._stream()
        d = torch.zeros(self.NK * self.NJ * self.NI, dtype=torch.float64, device=self.device)
        _check(lib().fg_op_diagonal(self.op.handle, d.data_ptr(), 1, DEVICE))
        out = torch.zeros(self.NK, self.NJ, self.pitch, dtype=torch.float64, device=self.device)
        out[:, :, :self.NI] = d.view(self.NK, self.NJ, self.NI)
        return out.view(-1)

    # solver steps on native vectors, owned prefix [0, n_own) ------------
    def vec_dots(self, n_own, pairs, out):
        """out[j] = a_j . b_j over the owned prefix (device tensor out)."""
        self._stream()
        a = (C.c_void_p * 3)(*([pa.data_ptr() for pa, _ in pairs] + [None] * (3 - len(pairs))))
        b = (C.c_void_p * 3)(*([pb.data_ptr() for _, pb in pairs] + [None] * (3 - len(pairs))))
        _check(lib().fg_vec_dots(self.op.handle, int(n_own), len(pairs), a, b, out.data_ptr()))

    def vec_pcg_update(self, n_own, x, r, p, ap, dinv, z, rz_pap, rr_rz):
        self._stream()
        _check(lib().fg_vec_pcg_update(self.op.handle, int(n_own), x.data_ptr(), r.data_ptr(), p.data_ptr(),
                                       ap.data_ptr(), dinv.data_ptr(), z.data_ptr(), rz_pap.data_ptr(),
                                       rr_rz.data_ptr()))

    def vec_pupdate(self, z, p, num, den):
        self._stream()
        _check(lib().fg_vec_pupdate(self.op.handle, z.data_ptr(), p.data_ptr(), num.data_ptr(), den.data_ptr()))

    def close(self):
        self.op.close()


# ---------------------------------------------------------------------------
# sharded operator
# ---------------------------------------------------------------------------
class ShardedPAOperator:
    """PA operator of the global structured hex mesh, split into z slabs.

    ``mesh``/``order``/``kind``/``kappa``/``rho``/``ess_tags`` describe the
    GLOBAL problem exactly as for PAOperator (kappa/rho per quadrature point
    [E][qz][qy][qx] over all elements, or scalars); each rank keeps only its
    slab.  ``local_factory(mesh, order, kind, kappa, rho, c_mass, c_diff,
    ess_tags)`` builds the local operator (default GpuSlab)."""

    def __init__(self, comm: Comm, mesh, order, kind=DIFF, kappa=1.0, rho=1.0, c_mass=1.0, c_diff=1.0,
                 ess_tags=TAG_ALL, local_factory=None):
        if isinstance(mesh, dict):
            nx, ny, nz, vc = mesh["nx"], mesh["ny"], mesh["nz"], mesh.get("vcoord")
        else:
            (nx, ny, nz), vc = mesh, None
        self.comm, self.order = comm, int(order)
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.z0, self.z1 = slab_partition(self.nz, comm.size)[comm.rank]
        nzl, p, nq3 = self.z1 - self.z0, self.order, (self.order + 1) ** 3
        vcl = None
        if vc is not None:
            vcl = np.asarray(vc, dtype=np.float64).reshape(self.nz + 1, self.ny + 1, self.nx + 1, 3)
            vcl = np.ascontiguousarray(vcl[self.z0:self.z1 + 1]).reshape(-1, 3)

        def part(c):
            if np.isscalar(c):
                return c
            c = np.asarray(c, dtype=np.float64).reshape(self.nz, self.ny * self.nx * nq3)
            return np.ascontiguousarray(c[self.z0:self.z1]).ravel()

        first, last = comm.rank == 0, comm.rank == comm.size - 1
        tags = ess_tags & (TAG_X0 | TAG_X1 | TAG_Y0 | TAG_Y1)
        tags |= (ess_tags & TAG_Z0) if first else 0
        tags |= (ess_tags & TAG_Z1) if last else 0
        self.local_tags = tags
        factory = local_factory or GpuSlab
        self.local = factory(dict(nx=self.nx, ny=self.ny, nz=nzl, vcoord=vcl), p, kind, part(kappa), part(rho),
                             c_mass, c_diff, tags)
        L = self.local
        self.NI, self.NJ, self.NK, self.pitch = L.NI, L.NJ, L.NK, L.pitch
        self.K0 = self.z0 * p  # global index of local plane 0
        self.plane = self.NJ * self.pitch
        self.n_local = self.NK * self.plane
        self.n_own = self.n_local - (0 if last else self.plane)
        dev = getattr(L, "device", torch.device("cpu"))
        keep = torch.ones(self.NJ, self.pitch, dtype=torch.float64)
        keep[:, self.NI:] = 0.0
        if tags & TAG_X0:
            keep[:, 0] = 0.0
        if tags & TAG_X1:
            keep[:, self.NI - 1] = 0.0
        if tags & TAG_Y0:
            keep[0, :] = 0.0
        if tags & TAG_Y1:
            keep[self.NJ - 1, :] = 0.0
        self.keep = keep.view(-1).to(dev)
        self.device = dev

    # vectors ------------------------------------------------------------
    def zeros(self):
        return torch.zeros(self.n_local, dtype=torch.float64, device=self.device)

    def scatter(self, v_global):
        """The rank's local vector (native layout) of a global plain vector."""
        NIg, NJg = self.nx * self.order + 1, self.ny * self.order + 1
        v = np.asarray(v_global, dtype=np.float64).reshape(-1, NJg, NIg)[self.K0:self.K0 + self.NK]
        out = np.zeros((self.NK, self.NJ, self.pitch))
        out[:, :, :self.NI] = v
        return torch.from_numpy(out.ravel()).to(self.device)

    def owned(self, v_local):
        """The owned planes of a local vector as a plain numpy array (in
        global plane order; concatenating the ranks' pieces gives the global
        vector)."""
        nk = self.n_own // self.plane
        return v_local[:self.n_own].view(nk, self.NJ, self.pitch)[:, :, :self.NI].cpu().numpy().ravel()

    # operator -----------------------------------------------------------
    def _halo_sum(self, y):
        size, rank = self.comm.size, self.comm.rank
        if size == 1:
            return y
        P = self.plane
        lo = y[:P].clone() if rank > 0 else None
        hi = y[self.n_local - P:].clone() if rank < size - 1 else None
        rlo, rhi = self.comm.exchange(lo, hi)
        if rlo is not None:
            y[:P] += rlo * self.keep
        if rhi is not None:
            y[self.n_local - P:] += rhi * self.keep
        return y

    def apply(self, x, y):
        """y = A x on consistent local vectors (x: both copies of each
        interface plane equal); the result is consistent."""
        self.local.apply(x, y)
        return self._halo_sum(y)

    def diagonal(self):
        return self._halo_sum(self.local.diagonal())

    def dots(self, pairs):
        """Global dots over owned DOFs (ParVector::global_dot), one
        allreduce for all pairs."""
        n = self.n_own
        t = torch.stack([torch.dot(a[:n], b[:n]) for a, b in pairs]).to(torch.float64)
        self.comm.allreduce_sum(t)
        return [float(v) for v in t.cpu()]

    def dot(self, a, b):
        return self.dots([(a, b)])[0]

    def close(self):
        if hasattr(self.local, "close"):
            self.local.close()


def par_solve_pcg_jacobi(A: ShardedPAOperator, b, x, cfg: SolverConfig | None = None) -> SolveResult:
    """Jacobi-preconditioned CG over the sharded operator, the iteration of
    par_solve_pcg_jacobi (par_solver.rs:262-342): same updates, same
    stopping rule (||r||/||b|| < rtol or ||r|| < atol), pap ~ 0 breaks off.
    The reference takes r.global_dot(r) and r.global_dot(z) in separate
    reductions; here z = D^-1 r is formed first and both dots share one
    allreduce (same values).  b, x: consistent local vectors; x holds the
    guess on entry and the solution on exit."""
    cfg = cfg or SolverConfig()
    if hasattr(A.local, "vec_pcg_update"):
        return _pcg_jacobi_device(A, b, x, cfg)
    d = A.diagonal()
    inv = d.clone()
    big = d.abs() > 1e-30
    inv[big] = 1.0 / d[big]
    inv[~big] = 1.0
    ax = A.zeros()
    A.apply(x, ax)
    r = b - ax
    z = inv * r
    p = z.clone()
    rz, bb = A.dots([(r, z), (b, b)])
    b_norm = bb ** 0.5
    if b_norm < 1e-30:
        return SolveResult(True, 0, 0.0)
    ap = A.zeros()
    for it in range(cfg.max_iter):
        A.apply(p, ap)
        pap = A.dot(p, ap)
        if abs(pap) < 1e-30:
            break
        alpha = rz / pap
        x.add_(p, alpha=alpha)
        r.add_(ap, alpha=-alpha)
        torch.mul(inv, r, out=z)
        rr, rz_new = A.dots([(r, r), (r, z)])
        res = rr ** 0.5 / b_norm
        if res < cfg.rtol or rr ** 0.5 < cfg.atol:
            return SolveResult(True, it + 1, res, applies=it + 2)
        beta = rz_new / rz
        p.mul_(beta).add_(z)
        rz = rz_new
    rr = A.dot(r, r)
    return SolveResult(False, cfg.max_iter, rr ** 0.5 / b_norm, applies=cfg.max_iter + 1)


def _pcg_jacobi_device(A: ShardedPAOperator, b, x, cfg: SolverConfig) -> SolveResult:
    """par_solve_pcg_jacobi with the vector work in the library's kernels
    (GPU slabs): the same iteration and stopping rule as the torch form
    above; the scalars live on the device and the host reads p.Ap (the
    breakdown test) and r.r (the stopping test) once per iteration, as the
    reference's loop does."""
    L, n_own = A.local, A.n_own
    d = A.diagonal()
    inv = torch.ones_like(d)
    big = d.abs() > 1e-30
    inv[big] = 1.0 / d[big]
    ax = A.zeros()
    A.apply(x, ax)
    r = b - ax
    z = inv * r
    p = z.clone()
    dev = r.device
    init = torch.zeros(2, dtype=torch.float64, device=dev)
    L.vec_dots(n_own, [(r, z), (b, b)], init)
    A.comm.allreduce_sum(init)
    b_norm = float(init[1]) ** 0.5
    if b_norm < 1e-30:
        return SolveResult(True, 0, 0.0)
    rz_pap = torch.zeros(2, dtype=torch.float64, device=dev)
    rr_rz = torch.zeros(2, dtype=torch.float64, device=dev)
    rz_pap[0:1].copy_(init[0:1])
    ap = A.zeros()
    for it in range(cfg.max_iter):
        A.apply(p, ap)
        L.vec_dots(n_own, [(p, ap)], rz_pap[1:2])
        A.comm.allreduce_sum(rz_pap[1:2])
        if abs(float(rz_pap[1])) < 1e-30:
            break
        L.vec_pcg_update(n_own, x, r, p, ap, inv, z, rz_pap, rr_rz)
        A.comm.allreduce_sum(rr_rz)
        rn = float(rr_rz[0]) ** 0.5
        res = rn / b_norm
        if res < cfg.rtol or rn < cfg.atol:
            return SolveResult(True, it + 1, res, applies=it + 2)
        L.vec_pupdate(z, p, rr_rz[1:2], rz_pap[0:1])
        rz_pap[0:1].copy_(rr_rz[1:2])
    rr = A.dot(r, r)
    return SolveResult(False, cfg.max_iter, rr ** 0.5 / b_norm, applies=cfg.max_iter + 1)
