"""The peer-store exchanges (slab.PeerExchange, pencil.PeerExchange) through
their real host path on one GPU:

* on a one-rank NCCL process group: the buffers' CUDA IPC handles exported
  and gathered (all_gather_object), the fences real stream synchronizations
  and barriers, the transposes the FFT passes' stores (at one rank the peer
  is the rank itself; no kernel waits on anything); three steps against the
  same steps with the buffer-copy exchanges: potential within 1e-6,
  velocities within 1e-6 relative L2 (the deposits' shared-memory atomics
  sum in no fixed order);
* on two gloo processes sharing the GPU: slab.PeerBuffers opens the other
  process's buffer by CUDA IPC, each process writes a pattern into the
  other's buffer, and after a barrier each finds the other's pattern in its
  own -- the mapping the peer stores go through between processes.

Each runs in spawned processes so that their process groups stay out of the
other tests.
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _run(port, decomp, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), NCCL_NVLS_ENABLE="0")
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "particle-mesh_b200"), os.path.join(root, "tests")]
    from datetime import timedelta
    import torch.distributed as dist
    from loader import load_package
    pm = load_package()
    try:
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60), device_id=dev)
        ng, nrow, dt = 64, 64, 0.1
        stream = torch.cuda.current_stream(dev)
        mass, cp = ng ** 3 / nrow ** 3, 4 * np.pi
        pos, vel = pm.zeldovich_ic(ng, nrow, -2.0, 0.5, seed=9, device="cuda:0")
        plan = pm.Plan(ng, "fp32", "spectral", 4, stream=stream, device=dev)
        cell, off = plan.split(*pos)
        v = [a.float() for a in vel]
        ids = torch.arange(nrow ** 3, dtype=torch.int32, device=dev)
        D = getattr(pm, decomp)
        out = []
        for peer in (False, True):
            if decomp == "slab":
                dec = D.Slab(ng, 1, 0, "spectral", 4, stream=stream, device=dev)
                (part,) = D.distribute(cell, off, v, ids, ng, 1, [0])
                ex = D.PeerExchange(dec) if peer else D.DistExchange()
            else:
                dec = D.Pencil(ng, 1, 1, 0, "spectral", 4, stream=stream, device=dev)
                (part,) = D.distribute(cell, off, v, ids, ng, 1, 1, [0])
                ex = D.PeerExchange(dec, 1, 1) if peer else D.LocalExchange()
            for _ in range(3):
                D.step([dec], [part], ex, mass, cp, dt, dt)
            dec.check()
            torch.cuda.synchronize()
            w = part.words[:, :part.n]
            w = w[:, torch.argsort(w[7])]
            out.append((dec.potential()[..., :ng].double().clone(), w[4:7].view(torch.float32).double().clone()))
            dec.close()
            del ex
        (p0, v0), (p1, v1) = out
        q.put((float((p1 - p0).norm() / p0.norm()), float((v1 - v0).norm() / v0.norm()), ""))
    except Exception as e:  # noqa: BLE001
        q.put((None, None, f"{type(e).__name__}: {e}"))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


@pytest.mark.parametrize("decomp", ["slab", "pencil"])
def test_peer_exchange_on_one_rank(decomp):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_run, args=(_free_port(), decomp, q))
    p.start()
    perr, verr, msg = q.get(timeout=600)
    p.join(timeout=120)
    assert not msg, msg
    assert perr < 1e-6 and verr < 1e-6, (perr, verr)


def _ipc_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "particle-mesh_b200"), os.path.join(root, "tests")]
    from datetime import timedelta
    import torch.distributed as dist
    from loader import load_package
    pm = load_package()
    msg = ""
    try:
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        slab = pm.slab.Slab(64, world, rank, "spectral", 4, device=dev)
        slab.recv.zero_()
        torch.cuda.synchronize()
        peers = pm.slab.PeerBuffers(slab.lib, dist, None, [slab.recv])
        other = 1 - rank
        theirs = pm.slab._view(peers.ptrs[0][other], slab.recv.numel(), torch.float32, dev)
        theirs.fill_(float(rank + 1))
        torch.cuda.synchronize()
        dist.barrier()
        got = slab.recv.unique().tolist()
        if got != [float(other + 1)]:
            msg = f"rank {rank} found {got[:4]} in its buffer"
        dist.barrier()
        peers.close()
        slab.close()
    except Exception as e:  # noqa: BLE001
        msg = f"{type(e).__name__}: {e}"
    q.put((rank, msg))
    if dist.is_initialized():
        dist.destroy_process_group()


def test_ipc_peer_buffers_between_two_processes():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ipc_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
    assert out == {0: "", 1: ""}, out
