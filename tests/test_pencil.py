"""The pencil decomposition's host logic on CPU: partition, the ghost rows and
their fold, the two sub-group transposes (uneven kz chunks), the potential
halo in x then y, and the particle migration of ``pencil.step`` through
``DistExchange`` on four gloo ranks (2 x 2), and through ``LocalExchange``
with 1 x 1, 1 x 4, 4 x 1 and 2 x 4 pencils in one process.

The per-pencil kernels are the CPU stand-in of tests/pencil_cpu.py (FP64
numpy, the CUDA kernels' buffer layouts); tests/test_pencil_gpu.py runs the
same steps through the CUDA kernels.  Checks:
  * every particle lives on exactly one rank, the one owning its (x, y)
    cell, before and after the steps, and particles did migrate;
  * four gloo ranks give bit for bit the state of the 2 x 2 pencils run in
    one process (the exchanges agree);
  * every decomposition matches the undecomposed mesh (1 x 1) and the x-slab
    stand-in within FFT rounding (1e-12 relative potential, 1e-6 velocity).
"""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from test_slab import CP, DT, NG, NROW, STEPS, _free_port, _paths, initial_state, state_by_id


def run_local(px, py, steps=STEPS):
    _paths()
    from loader import load_package
    from pencil_cpu import CpuPencil
    P = load_package().pencil
    _, _, cell, off, v, ids = initial_state()
    pens = [CpuPencil(NG, px, py, r) for r in range(px * py)]
    parts = P.distribute(cell, off, v, ids, NG, px, py, range(px * py), cap_factor=3.0)
    mass = NG ** 3 / NROW ** 3
    for _ in range(steps):
        P.step(pens, parts, P.LocalExchange(), mass, CP, DT, DT)
    return pens, parts


def mesh(pens):
    """The potential of all pencils assembled into [ng][ng][ng]."""
    phi = np.zeros((NG, NG, NG))
    for q in pens:
        phi[q.x0:q.x0 + q.nx, q.y0:q.y0 + q.ny] = q.potential()[:, :, :NG].numpy()
    return phi


def _rank(rank, world, port, q, px, py):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    _paths()
    from datetime import timedelta
    from loader import load_package
    from pencil_cpu import CpuPencil
    P = load_package().pencil
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    _, _, cell, off, v, ids = initial_state()
    s = CpuPencil(NG, px, py, rank)
    (part,) = P.distribute(cell, off, v, ids, NG, px, py, [rank])
    n0 = part.n
    own0 = bool(torch.all(P.owner_of(part.cell[:part.n], NG, px, py) == rank))
    ex = P.DistExchange(px, py)
    mass = NG ** 3 / NROW ** 3
    for _ in range(STEPS):
        P.step([s], [part], ex, mass, CP, DT, DT)
    own1 = bool(torch.all(P.owner_of(part.cell[:part.n], NG, px, py) == rank))
    q.put((rank, n0, part.n, own0, own1, part.words[:, :part.n].clone().numpy(),
           s.potential()[:, :, :NG].clone().numpy(), s.x0, s.y0))
    dist.barrier()
    dist.destroy_process_group()


def test_four_gloo_ranks_match_one_process():
    px, py = 2, 2
    world = px * py
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q, px, py)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(o[3] and o[4] for o in out)
    assert sum(o[1] for o in out) == NROW ** 3 == sum(o[2] for o in out)
    assert any(o[1] != o[2] for o in out), "no particle migrated"
    w = np.concatenate([o[5] for o in out], axis=1)
    w = w[:, np.argsort(w[7])]
    assert np.array_equal(w[7], np.arange(NROW ** 3))
    pens2, parts2 = run_local(px, py)
    assert np.array_equal(w, state_by_id(parts2).numpy())
    for o, pq in zip(out, pens2):
        assert (o[7], o[8]) == (pq.x0, pq.y0)
        assert np.array_equal(o[6], pq.potential()[:, :, :NG].numpy())


@pytest.mark.parametrize("px,py", [(1, 4), (4, 1), (2, 4)])
def test_local_pencils_match_one(px, py):
    pens, parts = run_local(px, py, steps=2)
    pens1, parts1 = run_local(1, 1, steps=2)
    phi, phi1 = mesh(pens), mesh(pens1)
    assert np.linalg.norm(phi - phi1) / np.linalg.norm(phi1) < 1e-12
    w, w1 = state_by_id(parts).numpy(), state_by_id(parts1).numpy()
    v, v1 = w[4:7].view(np.float32).astype(np.float64), w1[4:7].view(np.float32).astype(np.float64)
    assert np.linalg.norm(v - v1) / np.linalg.norm(v1) < 1e-6
    _paths()
    from loader import load_package
    P = load_package().pencil
    for s, q in zip(pens, parts):
        assert bool(torch.all(P.owner_of(q.cell[:q.n], NG, px, py) == s.rank))


def test_one_pencil_matches_one_slab():
    from test_slab import potential, run_local as run_slab
    pens1, parts1 = run_local(1, 1, steps=2)
    slabs1, sparts1 = run_slab(1, steps=2)
    phi, phis = mesh(pens1), potential(slabs1).numpy()
    assert np.linalg.norm(phi - phis) / np.linalg.norm(phis) < 1e-12
    w, ws = state_by_id(parts1).numpy(), state_by_id(sparts1).numpy()
    v, vs = w[4:7].view(np.float32).astype(np.float64), ws[4:7].view(np.float32).astype(np.float64)
    assert np.linalg.norm(v - vs) / np.linalg.norm(vs) < 1e-6


def test_owner_and_splits():
    _paths()
    from loader import load_package
    from pencil_cpu import CpuPencil
    P = load_package().pencil
    # kz chunks of the 17 planes of a 32 mesh over 4 ranks: 4, 4, 4, 5
    q = CpuPencil(32, 2, 4, 3)
    assert [P.kbound(17, 4, c) for c in range(5)] == [0, 4, 8, 12, 17]
    send, recv = P.y_splits(q, True)
    assert send == [2 * 16 * 8 * h for h in (4, 4, 4, 5)] and recv == [2 * 16 * 8 * 5] * 4
    assert P.y_splits(q, False) == (recv, send)
    assert sum(send) <= q.send.numel() and sum(recv) <= q.recv.numel()
    assert sum(P.x_splits(q)) <= q.send.numel()
    cell = torch.tensor([(i << 20) | (j << 10) for i, j in ((0, 0), (15, 7), (16, 8), (31, 31))], dtype=torch.int32)
    assert P.owner_of(cell, 32, 2, 4).tolist() == [0, 0, 5, 7]


def _peer_rank(rank, world, port, q, px, py, bufs_a, bufs_b):
    """One rank of the peer-store transposes: its CpuPencil stores into the
    group members' buffers (shared-memory tensors standing in for peer-mapped
    device memory); the exchange's fences are gloo barriers."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    _paths()
    from datetime import timedelta
    from loader import load_package
    from pencil_cpu import CpuPencil
    P = load_package().pencil

    class SharedPeerExchange(P._PencilPeerTransposes, P.DistExchange):
        def __init__(self):
            P.DistExchange.__init__(self, px, py)
            self.a, self.b = bufs_a, bufs_b

        def fence(self):
            self.dist.barrier()

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    _, _, cell, off, v, ids = initial_state()
    s = CpuPencil(NG, px, py, rank)
    (part,) = P.distribute(cell, off, v, ids, NG, px, py, [rank])
    ex = SharedPeerExchange()
    mass = NG ** 3 / NROW ** 3
    for _ in range(STEPS):
        P.step([s], [part], ex, mass, CP, DT, DT)
    q.put((rank, part.words[:, :part.n].clone().numpy(), s.potential()[:, :, :NG].clone().numpy()))
    dist.barrier()
    dist.destroy_process_group()


def test_peer_store_transposes_on_four_gloo_ranks():
    """The pencil's fused-transpose protocol (pencil._PencilPeerTransposes:
    every pass stores into the group members' buffers, two buffers per rank
    alternating, fences between the phases) on 2 x 2 processes gives bit for
    bit the state of the all-to-all transposes."""
    px, py = 2, 2
    world = px * py
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    n = _xfer_floats(NG, px, py)
    bufs_a = [torch.zeros(n, dtype=torch.float64).share_memory_() for _ in range(world)]
    bufs_b = [torch.zeros(n, dtype=torch.float64).share_memory_() for _ in range(world)]
    procs = [ctx.Process(target=_peer_rank, args=(r, world, port, q, px, py, bufs_a, bufs_b)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    w = np.concatenate([o[1] for o in out], axis=1)
    w = w[:, np.argsort(w[7])]
    pens2, parts2 = run_local(px, py)
    assert np.array_equal(w, state_by_id(parts2).numpy())
    for o, pq in zip(out, pens2):
        assert np.array_equal(o[2], pq.potential()[:, :, :NG].numpy())


def _xfer_floats(ng, px, py):
    _paths()
    from pencil_cpu import CpuPencil
    return CpuPencil(ng, px, py, 0).send.numel()
