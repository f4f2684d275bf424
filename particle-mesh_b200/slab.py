"""x-slab decomposition of one periodic mesh over several GPUs.

The reference's own parallel layout: particles and mesh split over MPI ranks,
the FFT on x-slabs (FFTW-MPI ``local_n0``, src/fft/fftw/fft.cpp:16), the
density sent to the slab owners with its +1 ghost planes and folded there
(src/decomp/slab/transpose_slab.cpp:3-39, reorder_slab.cpp:43-68), the
spectrum transposed by FFTW-MPI (fft.cpp:96-97), the potential returned with
-1/+2 ghost planes (reorder_slab_back.cpp:37-49, transpose_slab_back.cpp:3-49).
Here every rank (one GPU) owns the x planes [r nx, (r + 1) nx) of the mesh
and the particles whose cell lies there, and one step is

    deposit (+ z R2C)  ghost plane -> r + 1, fold   y forward
    all-to-all         x + Green                    all-to-all
    y inverse, z C2R   potential halo (2 below, 3 above)
    gather + kick + drift                           particle migration

The per-slab work runs in this package's CUDA kernels (``pm_slab_*`` of the C
ABI); the exchanges belong to an ``Exchange``: ``DistExchange`` over
torch.distributed (NCCL between GPUs; every rank takes the same collective
steps in the same order), or ``LocalExchange``, which holds every slab of the
decomposition in one process and moves the data with device copies (the
slabs run one after another; nothing waits on another slab's kernel).
``PeerExchange`` / ``LocalPeerExchange`` replace the two spectrum all-to-alls
by the FFT passes' own stores into the other ranks' buffers (mapped by CUDA
IPC; a barrier between the phases).  ``step`` is written once
against all of them.

Particles: split positions (cell word, three FP32 offsets), FP32
velocities, and a 32-bit particle id, held per rank in ``SlabParticles``
with spare capacity for arrivals.  Migration after the drift is new: the
reference never moves particles.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib as L
from ._lib import PMError, check
from .pm import _GREEN, _vp

WORDS = 8  # cell, ox, oy, oz, vx, vy, vz, id


def _view(ptr: int, numel: int, dtype, device) -> torch.Tensor:
    """A flat tensor over device memory owned by a slab (valid while it lives)."""
    class _Arr:
        __cuda_array_interface__ = {"shape": (numel,), "typestr": {torch.float32: "<f4", torch.int32: "<i4"}[dtype],
                                    "data": (ptr, False), "version": 3, "strides": None}
    return torch.as_tensor(_Arr(), device=device)


class SlabParticles:
    """One rank's particles: WORDS arrays of 32-bit words with capacity `cap`,
    the first `n` entries live.  Offsets and velocities are float32 views of
    the same storage as the words."""

    def __init__(self, cap: int, device):
        self.cap, self.n = int(cap), 0
        self.words = torch.zeros((WORDS, self.cap), dtype=torch.int32, device=device)

    @property
    def cell(self):
        return self.words[0]

    @property
    def off(self):
        return [self.words[1 + a].view(torch.float32) for a in range(3)]

    @property
    def vel(self):
        return [self.words[4 + a].view(torch.float32) for a in range(3)]

    @property
    def ids(self):
        return self.words[7]

    def arrays(self):
        return [self.words[w] for w in range(WORDS)]

    def set(self, cell, off, vel, ids):
        n = cell.numel()
        if n > self.cap:
            raise PMError(L.PM_ERR_SIZE, f"{n} particles exceed the slab capacity {self.cap}")
        self.words[0, :n] = cell
        for a in range(3):
            self.words[1 + a, :n] = off[a].view(torch.int32)
            self.words[4 + a, :n] = vel[a].view(torch.int32)
        self.words[7, :n] = ids
        self.n = n


def owner_of(cell: torch.Tensor, ng: int, nranks: int) -> torch.Tensor:
    """Rank owning each particle: its x cell (bits 20..29 of the cell word) // nx."""
    return ((cell.to(torch.int64) >> 20) % ng) // (ng // nranks)


class Slab:
    """One rank's x-slab: geometry, device buffers and the per-slab kernels."""

    def __init__(self, ng: int, nranks: int, rank: int, green: str = "spectral", grad_order: int = 4,
                 stream: torch.cuda.Stream | None = None, device=None):
        self.lib = L.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.ng, self.nranks, self.rank = ng, nranks, rank
        with torch.cuda.device(self.device):
            self.stream = stream if stream is not None else torch.cuda.current_stream(self.device)
            h = ctypes.c_void_p()
            check(self.lib.pm_slab_create(ng, nranks, rank, _GREEN[green], grad_order,
                                          ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self._h = h
        nx, x0 = ctypes.c_int(), ctypes.c_int()
        pf, xf, nb = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
        buf, send, recv = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(self.lib.pm_slab_info(h, ctypes.byref(nx), ctypes.byref(x0), ctypes.byref(pf), ctypes.byref(buf),
                                    ctypes.byref(send), ctypes.byref(recv), ctypes.byref(xf), ctypes.byref(nb)))
        self.nx, self.x0, self.plane = nx.value, x0.value, pf.value
        self.buf = _view(buf.value, (self.nx + 6) * self.plane, torch.float32, self.device).view(
            self.nx + 6, ng, ng + 2)
        self.send = _view(send.value, xf.value, torch.float32, self.device)
        self.recv = _view(recv.value, xf.value, torch.float32, self.device)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.pm_slab_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    # buffer planes the exchanges move (see include/pm_b200.h)
    def ghost_plane(self):
        return self.buf[self.nx + 2]

    def potential(self):
        """The own planes [nx][ng][ng + 2] (the potential after backward())."""
        return self.buf[2:self.nx + 2]

    def check(self):
        check(self.lib.pm_slab_check(self._h))

    def plan_handle(self):
        """The slab's pm_plan (stage timers, stream)."""
        h = ctypes.c_void_p()
        check(self.lib.pm_slab_plan(self._h, ctypes.byref(h)))
        return h

    def set_timing(self, on: bool = True):
        check(self.lib.pm_plan_set_timing(self.plan_handle(), 1 if on else 0))

    def read_timing(self, reset: bool = True) -> dict:
        """{stage: (milliseconds, launches)} of the slab's kernels since the last reset."""
        ms = (ctypes.c_double * L.STAGE_COUNT)()
        n = (ctypes.c_int64 * L.STAGE_COUNT)()
        check(self.lib.pm_plan_read_timing(self.plan_handle(), ms, n, 1 if reset else 0))
        return {self.lib.pm_stage_name(i).decode(): (ms[i], n[i]) for i in range(L.STAGE_COUNT) if n[i]}

    def device_bytes(self) -> int:
        nb = ctypes.c_size_t()
        check(self.lib.pm_slab_info(self._h, None, None, None, None, None, None, None, ctypes.byref(nb)))
        return nb.value

    # per-slab kernels
    def deposit(self, q: SlabParticles, mass: float):
        off = q.off
        check(self.lib.pm_slab_deposit_f32(self._h, _vp(q.cell), *(_vp(t) for t in off), q.n, float(mass)))

    def fold(self, ghost: torch.Tensor):
        check(self.lib.pm_slab_fold_f32(self._h, _vp(ghost)))

    def forward(self):
        check(self.lib.pm_slab_forward_f32(self._h))

    def xgreen(self, c_poisson: float):
        check(self.lib.pm_slab_xgreen_f32(self._h, float(c_poisson)))

    def backward(self):
        check(self.lib.pm_slab_backward_f32(self._h))

    # transposes by peer stores (pm_slab_*_peers_f32): one device pointer per
    # rank, in rank order
    def forward_peers(self, peer_recv):
        arr = (ctypes.c_void_p * len(peer_recv))(*peer_recv)
        check(self.lib.pm_slab_forward_peers_f32(self._h, arr, len(peer_recv)))

    def xgreen_peers(self, recv_ptr: int, c_poisson: float, peer_rows):
        arr = (ctypes.c_void_p * len(peer_rows))(*peer_rows)
        check(self.lib.pm_slab_xgreen_peers_f32(self._h, ctypes.c_void_p(recv_ptr), float(c_poisson), arr,
                                                len(peer_rows)))

    def backward_rows(self, rows_ptr: int):
        check(self.lib.pm_slab_backward_rows_f32(self._h, ctypes.c_void_p(rows_ptr)))

    def kick_drift(self, q: SlabParticles, c_kick: float, dt: float):
        check(self.lib.pm_slab_kick_drift_f32(self._h, _vp(q.cell), *(_vp(t) for t in q.off),
                                              *(_vp(t) for t in q.vel), q.n, float(c_kick), float(dt)))

    def migrate_sort(self, q: SlabParticles) -> list[int]:
        counts = (ctypes.c_int64 * self.nranks)()
        check(self.lib.pm_slab_migrate_sort(self._h, _vp(q.cell), q.n, counts))
        return list(counts)

    def migrate_pack(self, q: SlabParticles, packed: torch.Tensor):
        arr = (ctypes.c_void_p * WORDS)(*(t.data_ptr() for t in q.arrays()))
        check(self.lib.pm_slab_migrate_pack(self._h, arr, WORDS, q.n, _vp(packed)))

    def migrate_unpack(self, packed: torch.Tensor, n: int, q: SlabParticles, at: int):
        if at + n > q.cap:
            raise PMError(L.PM_ERR_SIZE, f"{at + n} particles exceed the slab capacity {q.cap}")
        arr = (ctypes.c_void_p * WORDS)(*(t.data_ptr() for t in q.arrays()))
        check(self.lib.pm_slab_migrate_unpack(self._h, _vp(packed), n, arr, WORDS, at))


# ------------------------------------------------------------------ exchanges
class _Transposes:
    """The spectrum passes around the two global transposes, with the
    transposes as all-to-alls of the send / recv buffers."""

    def forward(self, slabs):
        for s in slabs:
            s.forward()
        self.alltoall(slabs)

    def xgreen(self, slabs, c_poisson):
        for s in slabs:
            s.xgreen(c_poisson)
        self.alltoall(slabs)

    def backward(self, slabs):
        for s in slabs:
            s.backward()


class LocalExchange(_Transposes):
    """Every slab of the decomposition in this process; the exchanges are
    device copies on the current stream, slab after slab."""

    def ghost(self, slabs):
        p = len(slabs)
        for r, s in enumerate(slabs):
            slabs[(r + 1) % p].fold(s.ghost_plane())

    def alltoall(self, slabs):
        p = len(slabs)
        for d, sd in enumerate(slabs):
            blk = sd.recv.numel() // p
            for r, sr in enumerate(slabs):
                sd.recv[r * blk:(r + 1) * blk].copy_(sr.send[d * blk:(d + 1) * blk])

    def halo(self, slabs):
        p = len(slabs)
        for r, s in enumerate(slabs):
            nx = s.nx
            slabs[(r + 1) % p].buf[0:2].copy_(s.buf[nx:nx + 2])
            slabs[(r - 1) % p].buf[nx + 2:nx + 5].copy_(s.buf[2:5])

    def migrate(self, slabs, parts):
        p = len(slabs)
        if p == 1:  # one slab holds the whole periodic mesh: nothing leaves it
            return
        groups = []
        for s, q in zip(slabs, parts):
            counts = s.migrate_sort(q)
            packed = torch.empty((max(q.n, 1), WORDS), dtype=torch.int32, device=q.words.device)
            s.migrate_pack(q, packed)
            starts = [sum(counts[:d]) for d in range(p)]
            groups.append([packed[starts[d]:starts[d] + counts[d]] for d in range(p)])
        for d, (s, q) in enumerate(zip(slabs, parts)):
            incoming = torch.cat([groups[r][d] for r in range(p)]) if p > 1 else groups[0][0].clone()
            s.migrate_unpack(incoming, incoming.shape[0], q, 0)
            q.n = incoming.shape[0]


class DistExchange(_Transposes):
    """This process's one slab; the exchanges are torch.distributed
    collectives (NCCL between GPUs, gloo on CPU tensors), taken by every rank
    in the same order."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group

    def _sendrecv(self, send_t, to, recv_t, frm):
        d = self.dist
        ops = [d.P2POp(d.isend, send_t, to, self.group), d.P2POp(d.irecv, recv_t, frm, self.group)]
        for w in d.batch_isend_irecv(ops):
            w.wait()

    def ghost(self, slabs):
        (s,) = slabs
        p, r = s.nranks, s.rank
        if p == 1:
            s.fold(s.ghost_plane())
            return
        tmp = torch.empty_like(s.ghost_plane())
        self._sendrecv(s.ghost_plane().contiguous(), (r + 1) % p, tmp, (r - 1) % p)
        s.fold(tmp)

    def alltoall(self, slabs):
        (s,) = slabs
        if s.nranks == 1:
            s.recv.copy_(s.send)
            return
        self.dist.all_to_all_single(s.recv, s.send, group=self.group)

    def halo(self, slabs):
        (s,) = slabs
        p, r, nx = s.nranks, s.rank, s.nx
        if p == 1:
            s.buf[0:2].copy_(s.buf[nx:nx + 2])
            s.buf[nx + 2:nx + 5].copy_(s.buf[2:5])
            return
        lo = torch.empty_like(s.buf[0:2])
        hi = torch.empty_like(s.buf[nx + 2:nx + 5])
        self._sendrecv(s.buf[nx:nx + 2].contiguous(), (r + 1) % p, lo, (r - 1) % p)
        self._sendrecv(s.buf[2:5].contiguous(), (r - 1) % p, hi, (r + 1) % p)
        s.buf[0:2].copy_(lo)
        s.buf[nx + 2:nx + 5].copy_(hi)

    def migrate(self, slabs, parts):
        (s,), (q,) = slabs, parts
        p = s.nranks
        if p == 1:  # one slab holds the whole periodic mesh: nothing leaves it
            return
        dev = q.words.device
        counts = s.migrate_sort(q)
        packed = torch.empty((max(q.n, 1), WORDS), dtype=torch.int32, device=dev)
        s.migrate_pack(q, packed)
        send_c = torch.tensor(counts, dtype=torch.int64, device=dev)
        recv_c = torch.empty_like(send_c)
        self.dist.all_to_all_single(recv_c, send_c, group=self.group)
        rc = [int(v) for v in recv_c.tolist()]
        total = sum(rc)
        if total > q.cap:
            raise PMError(L.PM_ERR_SIZE, f"{total} particles arrive at rank {s.rank}, capacity {q.cap}")
        incoming = torch.empty((max(total, 1), WORDS), dtype=torch.int32, device=dev)
        self.dist.all_to_all_single(incoming[:total], packed[:q.n], output_split_sizes=rc,
                                    input_split_sizes=counts, group=self.group)
        s.migrate_unpack(incoming, total, q, 0)
        q.n = total


class _PeerTransposes:
    """The two transposes as stores into the other ranks' buffers
    (pm_slab_forward_peers_f32, pm_slab_xgreen_peers_f32): `recv[r]` and
    `rows[r]` are the device addresses of rank r's two transpose buffers;
    `fence()` separates the phases across the ranks."""

    def forward(self, slabs):
        self.fence()  # every rank done reading its buffers of the last step
        for s in slabs:
            s.forward_peers(self.recv)
        self.fence()

    def xgreen(self, slabs, c_poisson):
        for s in slabs:
            s.xgreen_peers(self.recv[s.rank], c_poisson, self.rows)
        self.fence()

    def backward(self, slabs):
        for s in slabs:
            s.backward_rows(self.rows[s.rank])


class LocalPeerExchange(_PeerTransposes, LocalExchange):
    """LocalExchange with the transposes done by the kernels' stores into the
    other slabs' buffers (all in one process on one GPU: the slabs' own send
    / recv buffers; stream order separates the phases)."""

    def __init__(self, slabs):
        self.recv = [s.recv.data_ptr() for s in slabs]
        self.rows = [s.send.data_ptr() for s in slabs]

    def fence(self):
        pass


class PeerBuffers:
    """Every rank's copies of some of its own device buffers, mapped into this
    process: each rank exports its buffers with CUDA IPC (pm_ipc_export), the
    handles travel by all_gather_object, and each rank opens the others'
    (pm_ipc_open; its own by address).  Plain peer mappings: no multicast
    object is bound to the memory.  `ptrs[b][r]` is buffer b of rank r.
    Collective: every rank of the group constructs it at the same point."""

    def __init__(self, lib, dist, group, buffers):
        self.lib, self._opened = lib, []
        handles = []
        for t in buffers:
            h = ctypes.create_string_buffer(L.PM_IPC_HANDLE_BYTES)
            check(lib.pm_ipc_export(ctypes.c_void_p(t.data_ptr()), h))
            handles.append(h.raw)
        world = dist.get_world_size(group)
        me = dist.get_rank(group)
        allh = [None] * world
        dist.all_gather_object(allh, handles, group=group)
        self.ptrs = [[0] * world for _ in buffers]
        for r in range(world):
            for b, t in enumerate(buffers):
                if r == me:
                    self.ptrs[b][r] = t.data_ptr()
                else:
                    p = ctypes.c_void_p()
                    check(lib.pm_ipc_open(ctypes.create_string_buffer(allh[r][b], L.PM_IPC_HANDLE_BYTES),
                                          ctypes.byref(p)))
                    self._opened.append(p)
                    self.ptrs[b][r] = p.value

    def close(self):
        for p in self._opened:
            self.lib.pm_ipc_close(p)
        self._opened = []

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


class PeerExchange(_PeerTransposes, DistExchange):
    """DistExchange with the transposes done by the kernels' stores into the
    other GPUs' memory: every rank's own send / recv buffers mapped into
    every process by CUDA IPC (PeerBuffers; no multicast), a host-side
    barrier (stream synchronize, then dist.barrier) between the phases.
    Construct it on every rank at the same point (collective)."""

    def __init__(self, slab, group=None):
        DistExchange.__init__(self, group)
        self._peers = PeerBuffers(slab.lib, self.dist, group, [slab.recv, slab.send])
        self.recv, self.rows = self._peers.ptrs
        self._stream = slab.stream

    def fence(self):
        self._stream.synchronize()
        self.dist.barrier(group=self.group)

    def close(self):
        self._peers.close()


def step(slabs, parts, exchange, mass: float, c_poisson: float, c_kick: float, dt: float):
    """One PM step of a decomposed mesh: deposit, Poisson solve, gather +
    kick + drift, migration.  `slabs` / `parts` are every slab of the
    decomposition (LocalExchange) or this rank's one (DistExchange)."""
    step_potential(slabs, parts, exchange, mass, c_poisson)
    step_finish(slabs, parts, exchange, c_kick, dt)


def step_potential(slabs, parts, exchange, mass: float, c_poisson: float):
    """The first part of `step`: deposit, ghost fold, Poisson solve, potential
    halo.  Reads only the particles' cell and offset words (0-3)."""
    for s, q in zip(slabs, parts):
        s.deposit(q, mass)
    exchange.ghost(slabs)
    exchange.forward(slabs)
    exchange.xgreen(slabs, c_poisson)
    exchange.backward(slabs)
    exchange.halo(slabs)


def step_finish(slabs, parts, exchange, c_kick: float, dt: float):
    """The rest of `step`: gather + kick + drift, migration."""
    for s, q in zip(slabs, parts):
        s.kick_drift(q, c_kick, dt)
    exchange.migrate(slabs, parts)


def deal_boxes(particles_per_box, nranks: int):
    """Boxes of an ensemble dealt to ranks, largest first to the least loaded
    rank (independent boxes: no exchange).  Returns one box list per rank."""
    load = [0] * nranks
    out = [[] for _ in range(nranks)]
    for b in sorted(range(len(particles_per_box)), key=lambda b: (-particles_per_box[b], b)):
        r = min(range(nranks), key=lambda r: (load[r], r))
        out[r].append(b)
        load[r] += particles_per_box[b]
    return [sorted(o) for o in out]


def distribute(cell, off, vel, ids, ng: int, nranks: int, ranks, cap_factor: float = 1.5, device=None):
    """SlabParticles for each rank in `ranks`: the particles whose x cell lies
    in that rank's slab, with capacity cap_factor x the even share."""
    own = owner_of(cell, ng, nranks)
    share = (cell.numel() + nranks - 1) // nranks
    out = []
    for r in ranks:
        sel = torch.nonzero(own == r).flatten()
        q = SlabParticles(max(int(cap_factor * share), sel.numel()) + 64, device if device is not None else cell.device)
        q.set(cell[sel], [a[sel] for a in off], [a[sel] for a in vel], ids[sel])
        out.append(q)
    return out
