"""Sharded PA operator and Jacobi-PCG (femgpu.sharded) on CPU.

The z-slab partition, the halo sum of interface planes, the owned-DOF dots
and the distributed PCG of par_solve_pcg_jacobi (par_solver.rs:262-342) run
with gloo process ranks and with thread ranks.  The rank's local operator is
a test stand-in built on the oracle's constrained apply and diagonal; the
assembled results are compared with the oracle on the whole mesh."""
import os
import threading

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

import oracle as O  # noqa: E402
from femgpu import SolverConfig  # noqa: E402
from femgpu import sharded as S  # noqa: E402
from sharded_cases import check, problem, reference  # noqa: E402


class OracleSlab:
    """Local operator stand-in: CPU tensors in the plain layout (pitch NI)."""

    device = torch.device("cpu")

    def __init__(self, mesh, order, kind, kappa, rho, c_mass, c_diff, ess_tags):
        self.m = O.Mesh(mesh["nx"], mesh["ny"], mesh["nz"], order, vcoord=mesh["vcoord"])
        sk, sr = np.isscalar(kappa), np.isscalar(rho)
        self.coef = O.Coef(kind, c_m=c_mass, c_k=c_diff, kappa_q=None if sk else kappa,
                           kappa=kappa if sk else 1.0, rho_q=None if sr else rho, rho=rho if sr else 1.0)
        self.ess = O.ess_mask(self.m, ess_tags)
        self.NK, self.NJ, self.NI = self.m.shape
        self.pitch = self.NI

    def apply(self, x, y):
        y.copy_(torch.from_numpy(O.apply_constrained(self.m, self.coef, self.ess, x.numpy())))

    def diagonal(self):
        return torch.from_numpy(O.diagonal(self.m, self.coef, self.ess))


def rank_work(comm, mesh, p, kq, tags, x, b):
    A = S.ShardedPAOperator(comm, mesh, p, kappa=kq, ess_tags=tags, local_factory=OracleSlab)
    yl = A.zeros()
    A.apply(A.scatter(x), yl)
    dl = A.diagonal()
    xs = A.zeros()
    res = S.par_solve_pcg_jacobi(A, A.scatter(b), xs, SolverConfig(rtol=1e-10, max_iter=2000))
    return dict(rank=comm.rank, K0=A.K0, NK=A.NK, y=A.owned(yl), y_local=yl.numpy().copy(), d=A.owned(dl),
                x=A.owned(xs), it=res.iterations, conv=res.converged)


def test_slab_partition():
    assert S.slab_partition(7, 3) == [(0, 3), (3, 5), (5, 7)]
    assert S.slab_partition(4, 4) == [(0, 1), (1, 2), (2, 3), (3, 4)]
    assert S.slab_partition(5, 1) == [(0, 5)]
    with pytest.raises(ValueError):
        S.slab_partition(2, 3)


def _run_threads(world, mesh, p, kq, tags, ref):
    g = S.ThreadGroup(world, timeout=60)
    out, errs = [None] * world, []

    def body(r):
        try:
            out[r] = rank_work(g.comm(r), mesh, p, kq, tags, ref["x"], ref["b"])
        except Exception as e:  # noqa: BLE001
            errs.append(e)
            g.barrier.abort()

    th = [threading.Thread(target=body, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=120)
    assert not errs, errs
    return out


@pytest.mark.parametrize("world", [1, 3, 4])
def test_thread_ranks(world):
    mesh, p, kq = problem()
    ref = reference(mesh, p, kq, 63)
    check(_run_threads(world, mesh, p, kq, 63, ref), ref)


def test_thread_ranks_partial_tags():
    # z1 free (the last rank's top plane is a natural boundary), y1 essential
    tags = S.TAG_Z0 | S.TAG_Y1 | S.TAG_X0
    mesh, p, kq = problem(nx=4, ny=5, nz=6, p=1, seed=5)
    ref = reference(mesh, p, kq, tags)
    check(_run_threads(3, mesh, p, kq, tags, ref), ref)


def test_rank_failure_breaks_barrier():
    # a rank that fails before its first exchange must not hang the others
    g = S.ThreadGroup(2, timeout=5)
    seen = []

    def good():
        try:
            g.comm(0).allreduce_sum(torch.ones(1, dtype=torch.float64))
        except threading.BrokenBarrierError:
            seen.append("broken")

    def bad():
        g.barrier.abort()

    t0, t1 = threading.Thread(target=good), threading.Thread(target=bad)
    t0.start()
    t1.start()
    t0.join(timeout=30)
    t1.join(timeout=30)
    assert seen == ["broken"]


def _gloo_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mesh, p, kq = problem()
        ref = reference(mesh, p, kq, 63)
        q.put(rank_work(S.TorchComm(), mesh, p, kq, 63, ref["x"], ref["b"]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + (os.getpid() + 17 * world) % 1000
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=180) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    mesh, p, kq = problem()
    check(res, reference(mesh, p, kq, 63))


def _gloo_subgroup_worker(rank, world, port, q):
    # global ranks 1 and 2 form the group of a 2-rank sharded solve; rank 0
    # only takes part in creating the group
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sub = dist.new_group([1, 2])
        if rank in (1, 2):
            mesh, p, kq = problem()
            ref = reference(mesh, p, kq, 63)
            q.put(rank_work(S.TorchComm(sub), mesh, p, kq, 63, ref["x"], ref["b"]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_non_default_group():
    """TorchComm on a subgroup: the plane exchange addresses its neighbours
    by global rank (dist.get_global_rank), so a group that does not start at
    global rank 0 gives the same answer as the default group."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29650 + os.getpid() % 1000
    procs = [ctx.Process(target=_gloo_subgroup_worker, args=(r, 3, port, q)) for r in range(3)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=180) for _ in range(2)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    mesh, p, kq = problem()
    check(res, reference(mesh, p, kq, 63))
