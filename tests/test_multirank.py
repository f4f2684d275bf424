"""Multi-GPU host logic on CPU ranks (gloo, world size 2): every rank runs its
own box (distinct seeds), the timed region is the max over ranks, and the
whole-job throughput counts every rank's particles.  No data-path
collective exists to test: boxes are independent."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    local_ms = 100.0 + 50.0 * rank
    t = bench.reduce_max(local_ms, world, "cpu")
    v = bench.throughput(world, 1000, 10, t)
    q.put((rank, t, v, bench.rank_seed(rank)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_timing_and_seeds():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(t == pytest.approx(150.0) for _, t, _, _ in out)
    assert all(v == pytest.approx(2 * 1000 * 10 / 0.150) for _, _, v, _ in out)
    assert len({s for _, _, _, s in out}) == world
