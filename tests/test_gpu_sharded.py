"""Sharded PA operator and Jacobi-PCG with the CUDA slab operator.

Ranks run as threads of this process on cuda:0, each with its own stream;
their kernels never wait on one another (the exchanges and sums meet on the
host), so one GPU carries them.  A one-rank NCCL group checks the
torch.distributed path.  Everything is compared with the oracle on the whole
mesh: assembled apply and diagonal <= 1e-12, PCG iterations within 1.  The
PCG's dots and vector updates run in the library's kernels (fg_vec_dots,
fg_vec_pcg_update, fg_vec_pupdate) with the scalars on the device."""
import os
import threading

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import femgpu  # noqa: E402
from femgpu import SolverConfig  # noqa: E402
from femgpu import sharded as S  # noqa: E402
from sharded_cases import check, problem, reference  # noqa: E402

pytestmark = pytest.mark.gpu


def _rank_work(A, x, b):
    assert hasattr(A.local, "vec_pcg_update")  # the PCG's vector work runs in the library's kernels
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        yl = A.zeros()
        A.apply(A.scatter(x), yl)
        dl = A.diagonal()
        xs = A.zeros()
        res = S.par_solve_pcg_jacobi(A, A.scatter(b), xs, SolverConfig(rtol=1e-10, max_iter=2000))
        NJ, NI = A.NJ, A.NI
        y_local = yl.view(A.NK, NJ, A.pitch)[:, :, :NI].cpu().numpy().ravel()
        return dict(rank=A.comm.rank, K0=A.K0, NK=A.NK, y=A.owned(yl), y_local=y_local, d=A.owned(dl),
                    x=A.owned(xs), it=res.iterations, conv=res.converged)


def _threads(world, mesh, p, kq, tags, ref):
    torch.cuda.set_device(0)
    g = S.ThreadGroup(world, timeout=120)
    ops = [S.ShardedPAOperator(g.comm(r), mesh, p, kappa=kq, ess_tags=tags) for r in range(world)]
    for A in ops:  # first launches (attributes, tables) from one thread
        A.local.apply(A.zeros(), A.zeros())
    torch.cuda.synchronize()
    out, errs = [None] * world, []

    def body(r):
        try:
            torch.cuda.set_device(0)
            out[r] = _rank_work(ops[r], ref["x"], ref["b"])
        except Exception as e:  # noqa: BLE001
            errs.append(e)
            g.barrier.abort()

    th = [threading.Thread(target=body, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    for A in ops:
        A.close()
    assert not errs, errs
    return out


@pytest.mark.parametrize("world,p,dims", [(2, 2, (12, 10, 14)), (3, 2, (20, 18, 24)), (4, 1, (33, 9, 10)),
                                          (3, 3, (8, 8, 9))])
def test_gpu_thread_ranks(world, p, dims):
    mesh, p, kq = problem(*dims, p=p, seed=7)
    ref = reference(mesh, p, kq, 63)
    check(_threads(world, mesh, p, kq, 63, ref), ref, 1e-12)


def test_gpu_thread_ranks_partial_tags():
    tags = S.TAG_Z0 | S.TAG_Y1 | S.TAG_X0
    mesh, p, kq = problem(10, 12, 9, p=2, seed=9)
    ref = reference(mesh, p, kq, tags)
    check(_threads(3, mesh, p, kq, tags, ref), ref, 1e-12)


def test_gpu_sharded_matches_single_operator():
    # the 1-rank sharded solve is the single-operator Jacobi PCG (fg_pcg)
    mesh, p, kq = problem(16, 12, 10, p=2, seed=4)
    ref = reference(mesh, p, kq, 63)
    out = _threads(1, mesh, p, kq, 63, ref)[0]
    op = femgpu.PADiffusionOperator(mesh, p, kappa=kq)
    xs = np.zeros(op.n_dofs())
    res = femgpu.solve_pcg_jacobi(op, ref["b"], xs, SolverConfig(rtol=1e-10, max_iter=2000))
    assert abs(res.iterations - out["it"]) <= 1
    assert np.linalg.norm(out["x"] - xs) <= 1e-8 * np.linalg.norm(xs)


def test_gpu_nccl_one_rank():
    import torch.distributed as dist

    torch.cuda.set_device(0)
    port = 29900 + os.getpid() % 500
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        mesh, p, kq = problem(9, 7, 8, p=2, seed=2)
        ref = reference(mesh, p, kq, 63)
        A = S.ShardedPAOperator(S.TorchComm(), mesh, p, kappa=kq)
        out = _rank_work(A, ref["x"], ref["b"])
        A.close()
        check([out], ref, 1e-12)
    finally:
        dist.destroy_process_group()
