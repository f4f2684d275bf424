"""The x-slab decomposition's host logic on CPU: partition, ghost fold, the
global transposes, the potential halo and the particle migration of
``slab.step`` through ``DistExchange`` on two gloo ranks, and through
``LocalExchange`` with 1, 2 and 4 slabs in one process.

The per-slab kernels are the CPU stand-in of tests/slab_cpu.py (FP64 numpy,
the CUDA kernels' buffer layouts); tests/test_slab_gpu.py runs the same steps
through the CUDA kernels.  Checks:
  * every particle lives on exactly one rank, the one owning its x cell,
    before and after the steps, and particles did migrate;
  * two gloo ranks give bit for bit the state of the two slabs run in one
    process (the exchanges agree);
  * 2 and 4 slabs match 1 slab (the decomposition changes no result beyond
    FFT rounding: 1e-12 relative on the potential, 1e-10 on velocities);
  * the first step's kick equals the oracle's forces (relative L2 1e-6: the
    split positions carry FP32 offsets).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

NG, NROW, STEPS, DT, CP = 32, 32, 4, 0.5, 4 * np.pi


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _paths():
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "particle-mesh_b200"), os.path.join(root, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)


def initial_state():
    _paths()
    from oracle import oracle as O
    from slab_cpu import pack_cell, split1
    pos, vel = O.zeldovich_ic(NG, NROW, -2.0, 0.5, seed=17)
    cells, offs = zip(*(split1(p, NG) for p in pos))
    cell = torch.from_numpy(pack_cell(*cells).view(np.int32).copy())
    off = [torch.from_numpy(o.copy()) for o in offs]
    v = [torch.from_numpy(a.astype(np.float32)) for a in vel]
    ids = torch.arange(NROW ** 3, dtype=torch.int32)
    return pos, vel, cell, off, v, ids


def run_local(nranks, steps=STEPS):
    _paths()
    from loader import load_package
    from slab_cpu import CpuSlab
    S = load_package().slab
    _, _, cell, off, v, ids = initial_state()
    slabs = [CpuSlab(NG, nranks, r) for r in range(nranks)]
    parts = S.distribute(cell, off, v, ids, NG, nranks, range(nranks))
    mass = NG ** 3 / NROW ** 3
    for _ in range(steps):
        S.step(slabs, parts, S.LocalExchange(), mass, CP, DT, DT)
    return slabs, parts


def state_by_id(parts):
    w = torch.cat([q.words[:, :q.n] for q in parts], dim=1)
    order = torch.argsort(w[7])
    return w[:, order]


def potential(slabs):
    return torch.cat([s.potential()[:, :, :NG] for s in slabs])


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    _paths()
    from datetime import timedelta
    from loader import load_package
    from slab_cpu import CpuSlab
    S = load_package().slab
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    _, _, cell, off, v, ids = initial_state()
    s = CpuSlab(NG, world, rank)
    (part,) = S.distribute(cell, off, v, ids, NG, world, [rank])
    n0 = part.n
    own0 = bool(torch.all(S.owner_of(part.cell[:part.n], NG, world) == rank))
    ex = S.DistExchange()
    mass = NG ** 3 / NROW ** 3
    for _ in range(STEPS):
        S.step([s], [part], ex, mass, CP, DT, DT)
    own1 = bool(torch.all(S.owner_of(part.cell[:part.n], NG, world) == rank))
    q.put((rank, n0, part.n, own0, own1, part.words[:, :part.n].clone().numpy(), s.potential()[:, :, :NG].clone().numpy()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_match_one_process_and_one_slab():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # partition: every particle on its owner, before and after, and some moved
    assert all(o[3] and o[4] for o in out)
    assert sum(o[1] for o in out) == NROW ** 3 == sum(o[2] for o in out)
    assert any(o[1] != o[2] for o in out), "no particle migrated; the test needs motion across slab faces"
    w = np.concatenate([o[5] for o in out], axis=1)
    w = w[:, np.argsort(w[7])]
    assert np.array_equal(w[7], np.arange(NROW ** 3))
    phi = np.concatenate([o[6] for o in out])
    # the same decomposition in one process: identical bits
    slabs2, parts2 = run_local(2)
    assert np.array_equal(w, state_by_id(parts2).numpy())
    assert np.array_equal(phi, potential(slabs2).numpy())
    # one slab: the undecomposed mesh
    slabs1, parts1 = run_local(1)
    w1 = state_by_id(parts1).numpy()
    phi1 = potential(slabs1).numpy()
    assert np.linalg.norm(phi - phi1) / np.linalg.norm(phi1) < 1e-12
    v, v1 = w[4:7].view(np.float32).astype(np.float64), w1[4:7].view(np.float32).astype(np.float64)
    assert np.linalg.norm(v - v1) / np.linalg.norm(v1) < 1e-6
    assert np.mean(w[0] != w1[0]) < 1e-3  # cells agree but for rounding at a face


def test_four_local_slabs_match_one():
    slabs4, parts4 = run_local(4, steps=2)
    slabs1, parts1 = run_local(1, steps=2)
    phi4, phi1 = potential(slabs4).numpy(), potential(slabs1).numpy()
    assert np.linalg.norm(phi4 - phi1) / np.linalg.norm(phi1) < 1e-12
    w4, w1 = state_by_id(parts4).numpy(), state_by_id(parts1).numpy()
    v4, v1 = w4[4:7].view(np.float32).astype(np.float64), w1[4:7].view(np.float32).astype(np.float64)
    assert np.linalg.norm(v4 - v1) / np.linalg.norm(v1) < 1e-6
    for s, q in zip(slabs4, parts4):
        _paths()
        from loader import load_package
        assert bool(torch.all(load_package().slab.owner_of(q.cell[:q.n], NG, 4) == s.rank))


def test_first_kick_matches_oracle_forces():
    _paths()
    from oracle import oracle as O
    pos, vel, *_ = initial_state()
    slabs, parts = run_local(2, steps=1)
    w = state_by_id(parts).numpy()
    v = w[4:7].view(np.float32).astype(np.float64)
    f = [np.zeros(NROW ** 3) for _ in range(3)]
    O.force_step(NG, *(a.copy() for a in pos), *f, NG ** 3 / NROW ** 3, CP, 1.0, 1, 4)
    kick = v - np.stack([a.astype(np.float32).astype(np.float64) for a in vel])
    err = np.linalg.norm(kick / DT - np.stack(f)) / np.linalg.norm(np.stack(f))
    assert err < 1e-5, err


def _peer_rank(rank, world, port, q, recv, rows):
    """One rank of the peer-store transposes: its CpuSlab stores into the
    other rank's buffers (shared-memory tensors standing in for peer-mapped
    device memory); the exchange's fences are gloo barriers."""
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

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    _, _, cell, off, v, ids = initial_state()
    s = CpuSlab(NG, world, rank)
    (part,) = S.distribute(cell, off, v, ids, NG, world, [rank])
    ex = SharedPeerExchange()
    mass = NG ** 3 / NROW ** 3
    for _ in range(STEPS):
        S.step([s], [part], ex, mass, CP, DT, DT)
    q.put((rank, part.words[:, :part.n].clone().numpy(), s.potential()[:, :, :NG].clone().numpy()))
    dist.barrier()
    dist.destroy_process_group()


def test_peer_store_transposes_on_two_gloo_ranks():
    """The fused-transpose protocol (slab._PeerTransposes: each rank's y
    forward and x + Green store straight into the other rank's buffers, fences
    between the phases) on two processes gives bit for bit the state of the
    all-to-all transposes."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    n = (NG // world) * NG * (NG + 2)
    recv = [torch.zeros(n, dtype=torch.float64).share_memory_() for _ in range(world)]
    rows = [torch.zeros(n, dtype=torch.float64).share_memory_() for _ in range(world)]
    procs = [ctx.Process(target=_peer_rank, args=(r, world, port, q, recv, rows)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    w = np.concatenate([o[1] for o in out], axis=1)
    w = w[:, np.argsort(w[7])]
    phi = np.concatenate([o[2] for o in out])
    slabs2, parts2 = run_local(2)
    assert np.array_equal(w, state_by_id(parts2).numpy())
    assert np.array_equal(phi, potential(slabs2).numpy())
