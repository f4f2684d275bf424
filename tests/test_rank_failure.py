"""Failure detection of the decomposed step on CPU (gloo ranks, no GPU): a
rank that leaves between two steps -- after its first step it exits without
taking part in any further collective -- must make the other rank's next
exchange end with an error inside the process group's timeout, not hang.
Run for the all-to-all transposes (slab.DistExchange) and for the
peer-store transposes (their fences are barriers), with the CPU stand-in of
the per-slab kernels.
"""
import os
import time

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from test_slab import CP, DT, NG, NROW, _free_port, _paths, initial_state

TIMEOUT_S = 10


def _rank(rank, world, port, q, peer, recv, rows):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    _paths()
    from datetime import timedelta
    from loader import load_package
    from slab_cpu import CpuSlab
    S = load_package().slab

    class SharedPeerExchange(S._PeerTransposes, S.DistExchange):
        def __init__(self):
            S.DistExchange.__init__(self)
            self.recv, self.rows = recv, rows

        def fence(self):
            self.dist.barrier()

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=TIMEOUT_S))
    _, _, cell, off, v, ids = initial_state()
    s = CpuSlab(NG, world, rank)
    (part,) = S.distribute(cell, off, v, ids, NG, world, [rank])
    ex = SharedPeerExchange() if peer else S.DistExchange()
    mass = NG ** 3 / NROW ** 3
    S.step([s], [part], ex, mass, CP, DT, DT)
    if rank == 1:
        _report(q, (rank, "left", 0.0))
        os._exit(0)  # leaves between steps: nothing of it is in flight
    t0 = time.monotonic()
    try:
        for _ in range(3):
            S.step([s], [part], ex, mass, CP, DT, DT)
        _report(q, (rank, "no error", time.monotonic() - t0))
    except Exception as e:  # noqa: BLE001
        _report(q, (rank, type(e).__name__, time.monotonic() - t0))
    os._exit(0)


def _report(q, item):
    """Put and flush (the process leaves with os._exit right after)."""
    q.put(item)
    q.close()
    q.join_thread()


@pytest.mark.parametrize("peer", [False, True])
def test_rank_leaving_between_steps_ends_the_others_exchange(peer):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    n = (NG // world) * NG * (NG + 2)
    recv = [torch.zeros(n, dtype=torch.float64).share_memory_() for _ in range(world)]
    rows = [torch.zeros(n, dtype=torch.float64).share_memory_() for _ in range(world)]
    procs = [ctx.Process(target=_rank, args=(r, world, port, q, peer, recv, rows)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict((r, (what, dt)) for r, what, dt in (q.get(timeout=120) for _ in range(world)))
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert out[1][0] == "left"
    what, elapsed = out[0]
    print(f"peer={peer}: rank 0 stopped with {what} after {elapsed:.2f} s")
    assert what != "no error", "the surviving rank stepped on without its peer"
    assert elapsed < 3 * TIMEOUT_S, elapsed
