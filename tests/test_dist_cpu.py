"""The bench's multi-rank path on CPU (gloo, world size 2): ranks read their
identity from the torchrun environment, every rank runs its own instance
(its own kappa seed), and timings are reduced to the slowest rank's before the
whole-job throughput is formed.  The path has no data-path collective: the
instances are independent (weak scaling, replicas)."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    from femgpu.fields import lognormal_kappa_q

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w, r, local = bench.dist_setup()
        t_ms = 10.0 + 5.0 * r  # rank 1 is the slow one
        t = bench.max_over_ranks(t_ms, w, torch.device("cpu"))
        kq = lognormal_kappa_q(4, 4, 4, 1, seed=r)
        out.put((r, w, local, t, bench.whole_job_gdofs(w, 1000, 10, t), float(np.asarray(kq).sum())))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 and r[2] == r[0] for r in res)
    assert all(r[3] == 15.0 for r in res)                      # slowest rank's time on every rank
    assert all(abs(r[4] - 2 * 1000 * 10 / 15e-3 / 1e9) < 1e-15 for r in res)
    assert res[0][5] != res[1][5]                               # independent instances
