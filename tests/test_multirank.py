"""Multi-GPU host logic on CPU ranks (gloo, world size 2): the timed region is
the max over ranks, the whole-job throughput counts every rank's particles,
and the ensemble's boxes are dealt to the ranks (disjoint, complete,
balanced).  The slab decomposition's exchanges are tested in test_slab.py."""
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
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "particle-mesh_b200")]
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    local_ms = 100.0 + 50.0 * rank
    t = bench.reduce_max(local_ms, world, "cpu")
    v = bench.throughput(world, 1000, 10, t)
    from loader import load_package
    S = load_package().slab
    sizes = [n ** 3 for n in (32, 48, 64, 96, 128, 32, 64, 128, 96, 48, 48)]
    mine = S.deal_boxes(sizes, world)[rank]
    q.put((rank, t, v, bench.rank_seed(rank), mine, sum(sizes[b] for b in mine)))
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
    assert all(o[1] == pytest.approx(150.0) for o in out)
    assert all(o[2] == pytest.approx(2 * 1000 * 10 / 0.150) for o in out)
    assert len({o[3] for o in out}) == world
    # ensemble boxes dealt to the ranks: disjoint, every box once, balanced
    dealt = [b for o in out for b in o[4]]
    assert sorted(dealt) == list(range(11))
    loads = [o[5] for o in out]
    assert max(loads) - min(loads) <= 128 ** 3
