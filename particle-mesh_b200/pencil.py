"""Pencil decomposition of one periodic mesh over px x py GPUs.

The reference names a pencil decomposition (``DECOMP_CHOICES`` lists
"pencil", Makefile:1) but ships only the x-slab one, whose FFT (FFTW-MPI,
src/fft/fftw/fft.cpp:11-16) caps the rank count at ng.  Here rank
r = rx py + ry (one GPU) owns the pencil x in [rx nx, (rx + 1) nx),
y in [ry ny, (ry + 1) ny), all z (nx = ng / px, ny = ng / py) and the
particles whose cell lies there.  One step:

    deposit          ghost rows -> (rx+1, ry), (rx, ry+1), (rx+1, ry+1); fold
    z R2C            all-to-all in the y group (kz chunks)    y forward
    all-to-all in the x group (ky chunks)    x forward, Green, x inverse
    all-to-all in the x group                y inverse
    all-to-all in the y group                z C2R
    potential halo (x rows, then y rows)     gather + kick + drift
    particle migration

The y group of a rank is the py ranks of its rx, the x group the px ranks of
its ry.  The per-pencil work runs in this package's CUDA kernels
(``pm_pencil_*`` of the C ABI); the exchanges belong to ``LocalExchange``
(every pencil in one process, device copies) or ``DistExchange``
(torch.distributed; NCCL sub-groups for the transposes), as for the slabs;
``PeerExchange`` / ``LocalPeerExchange`` do the four transposes as the FFT
passes' own stores into the group members' buffers.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib as L
from . import slab as _slab
from ._lib import PMError, check
from .pm import _GREEN, _vp
from .slab import WORDS, SlabParticles, _view


def kbound(h: int, py: int, c: int) -> int:
    """First kz plane of chunk c of the half spectrum's h planes over py ranks."""
    return (c * h) // py


def owner_of(cell: torch.Tensor, ng: int, px: int, py: int) -> torch.Tensor:
    """Rank owning each particle: (x cell // nx) py + (y cell // ny)."""
    c = cell.to(torch.int64)
    i, j = (c >> 20) % ng, ((c >> 10) & 1023) % ng
    return (i // (ng // px)) * py + j // (ng // py)


def y_splits(q, forward: bool):
    """(send sizes, recv sizes) in floats of the y-group transpose of pencil q,
    one entry per group member (ry order); blocks lie back to back."""
    blk = 2 * q.nx * q.ny
    hc = [kbound(q.h, q.py, c + 1) - kbound(q.h, q.py, c) for c in range(q.py)]
    mine = [blk * hc[q.ry]] * q.py
    other = [blk * hc[c] for c in range(q.py)]
    return (other, mine) if forward else (mine, other)


def x_splits(q):
    hc = kbound(q.h, q.py, q.ry + 1) - kbound(q.h, q.py, q.ry)
    return [2 * q.nx * q.nx * hc] * q.px


class Pencil:
    """One rank's pencil: geometry, device buffers and the per-pencil kernels."""

    def __init__(self, ng: int, px: int, py: int, rank: int, green: str = "spectral", grad_order: int = 4,
                 stream: torch.cuda.Stream | None = None, device=None):
        self.lib = L.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.ng, self.px, self.py, self.rank = ng, px, py, rank
        self.nranks, self.rx, self.ry, self.h = px * py, rank // py, rank % py, ng // 2 + 1
        with torch.cuda.device(self.device):
            self.stream = stream if stream is not None else torch.cuda.current_stream(self.device)
            h = ctypes.c_void_p()
            check(self.lib.pm_pencil_create(ng, px, py, rank, _GREEN[green], grad_order,
                                            ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self._h = h
        nx, ny, x0, y0 = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        xf, nb = ctypes.c_size_t(), ctypes.c_size_t()
        halo, send, recv = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(self.lib.pm_pencil_info(h, ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(x0), ctypes.byref(y0),
                                      ctypes.byref(halo), ctypes.byref(send), ctypes.byref(recv), ctypes.byref(xf),
                                      ctypes.byref(nb)))
        self.nx, self.ny, self.x0, self.y0 = nx.value, ny.value, x0.value, y0.value
        shape = (self.nx + 5, self.ny + 5, ng + 2)
        self.halo = _view(halo.value, shape[0] * shape[1] * shape[2], torch.float32, self.device).view(*shape)
        self.send = _view(send.value, xf.value, torch.float32, self.device)
        self.recv = _view(recv.value, xf.value, torch.float32, self.device)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.pm_pencil_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    # buffer rows the exchanges move (include/pm_b200.h)
    def xghost(self):
        return self.halo[self.nx + 2, 2:self.ny + 2]

    def yghost(self):
        return self.halo[2:self.nx + 2, self.ny + 2]

    def corner(self):
        return self.halo[self.nx + 2, self.ny + 2:self.ny + 3]

    def potential(self):
        """The own rows [nx][ny][ng + 2] (the potential after backward())."""
        return self.halo[2:self.nx + 2, 2:self.ny + 2]

    def check(self):
        check(self.lib.pm_pencil_check(self._h))

    def plan_handle(self):
        h = ctypes.c_void_p()
        check(self.lib.pm_pencil_plan(self._h, ctypes.byref(h)))
        return h

    def set_timing(self, on: bool = True):
        check(self.lib.pm_plan_set_timing(self.plan_handle(), 1 if on else 0))

    def read_timing(self, reset: bool = True) -> dict:
        ms = (ctypes.c_double * L.STAGE_COUNT)()
        n = (ctypes.c_int64 * L.STAGE_COUNT)()
        check(self.lib.pm_plan_read_timing(self.plan_handle(), ms, n, 1 if reset else 0))
        return {self.lib.pm_stage_name(i).decode(): (ms[i], n[i]) for i in range(L.STAGE_COUNT) if n[i]}

    def device_bytes(self) -> int:
        nb = ctypes.c_size_t()
        check(self.lib.pm_pencil_info(self._h, None, None, None, None, None, None, None, None, ctypes.byref(nb)))
        return nb.value

    # per-pencil kernels
    def deposit(self, q: SlabParticles, mass: float):
        check(self.lib.pm_pencil_deposit_f32(self._h, _vp(q.cell), *(_vp(t) for t in q.off), q.n, float(mass)))

    def fold(self, xghost: torch.Tensor, yghost: torch.Tensor, corner: torch.Tensor):
        for t in (xghost, yghost, corner):
            if not t.is_contiguous():
                raise PMError(L.PM_ERR_ARG, "ghost rows must be contiguous")
        check(self.lib.pm_pencil_fold_f32(self._h, _vp(xghost), _vp(yghost), _vp(corner)))

    def forward(self):
        check(self.lib.pm_pencil_forward_f32(self._h))

    def yfwd(self):
        check(self.lib.pm_pencil_yfwd_f32(self._h))

    def xgreen(self, c_poisson: float):
        check(self.lib.pm_pencil_xgreen_f32(self._h, float(c_poisson)))

    def yinv(self):
        check(self.lib.pm_pencil_yinv_f32(self._h))

    def backward(self):
        check(self.lib.pm_pencil_backward_f32(self._h))

    # transposes by peer stores (pm_pencil_*_peers_f32): peer buffer addresses
    # in group-member order, `inp` this rank's buffer the last phase filled
    @staticmethod
    def _ptrs(ptrs):
        return (ctypes.c_void_p * len(ptrs))(*ptrs), len(ptrs)

    def forward_peers(self, peer_a):
        check(self.lib.pm_pencil_forward_peers_f32(self._h, *self._ptrs(peer_a)))

    def yfwd_peers(self, inp: int, peer_b):
        check(self.lib.pm_pencil_yfwd_peers_f32(self._h, ctypes.c_void_p(inp), *self._ptrs(peer_b)))

    def xgreen_peers(self, inp: int, c_poisson: float, peer_a):
        check(self.lib.pm_pencil_xgreen_peers_f32(self._h, ctypes.c_void_p(inp), float(c_poisson),
                                                  *self._ptrs(peer_a)))

    def yinv_peers(self, inp: int, peer_b):
        check(self.lib.pm_pencil_yinv_peers_f32(self._h, ctypes.c_void_p(inp), *self._ptrs(peer_b)))

    def backward_from(self, inp: int):
        check(self.lib.pm_pencil_backward_from_f32(self._h, ctypes.c_void_p(inp)))

    def kick_drift(self, q: SlabParticles, c_kick: float, dt: float):
        check(self.lib.pm_pencil_kick_drift_f32(self._h, _vp(q.cell), *(_vp(t) for t in q.off),
                                                *(_vp(t) for t in q.vel), q.n, float(c_kick), float(dt)))

    def migrate_sort(self, q: SlabParticles) -> list[int]:
        counts = (ctypes.c_int64 * self.nranks)()
        check(self.lib.pm_pencil_migrate_sort(self._h, _vp(q.cell), q.n, counts))
        return list(counts)

    def migrate_pack(self, q: SlabParticles, packed: torch.Tensor):
        arr = (ctypes.c_void_p * WORDS)(*(t.data_ptr() for t in q.arrays()))
        check(self.lib.pm_pencil_migrate_pack(self._h, arr, WORDS, q.n, _vp(packed)))

    def migrate_unpack(self, packed: torch.Tensor, n: int, q: SlabParticles, at: int):
        if at + n > q.cap:
            raise PMError(L.PM_ERR_SIZE, f"{at + n} particles exceed the pencil capacity {q.cap}")
        arr = (ctypes.c_void_p * WORDS)(*(t.data_ptr() for t in q.arrays()))
        check(self.lib.pm_pencil_migrate_unpack(self._h, _vp(packed), n, arr, WORDS, at))


def _empty(t):
    """A contiguous buffer of t's shape (t may be a strided view)."""
    return torch.empty(t.shape, dtype=t.dtype, device=t.device)


def _rank(q, rx, ry):
    return (rx % q.px) * q.py + ry % q.py


# ------------------------------------------------------------------ exchanges
class _PencilTransposes:
    """The spectrum passes with the four transposes as all-to-alls of the
    send / recv buffers in the y and x groups."""

    def forward(self, pens):
        for p in pens:
            p.forward()
        self.ytrans(pens, True)

    def yfwd(self, pens):
        for p in pens:
            p.yfwd()
        self.xtrans(pens)

    def xgreen(self, pens, c_poisson):
        for p in pens:
            p.xgreen(c_poisson)
        self.xtrans(pens)

    def yinv(self, pens):
        for p in pens:
            p.yinv()
        self.ytrans(pens, False)

    def backward(self, pens):
        for p in pens:
            p.backward()


class _PencilPeerTransposes:
    """The four transposes as stores into the group members' buffers
    (pm_pencil_*_peers_f32): `a[r]`, `b[r]` are the device addresses of rank
    r's two transpose buffers, which alternate between the phases; `fence()`
    separates the phases across the ranks."""

    def _ygroup(self, q, bufs):
        return [bufs[q.rx * q.py + c] for c in range(q.py)]

    def _xgroup(self, q, bufs):
        return [bufs[d * q.py + q.ry] for d in range(q.px)]

    def forward(self, pens):
        self.fence()  # every rank done with its buffers of the last step
        for p in pens:
            p.forward_peers(self._ygroup(p, self.a))
        self.fence()

    def yfwd(self, pens):
        for p in pens:
            p.yfwd_peers(self.a[p.rank], self._xgroup(p, self.b))
        self.fence()

    def xgreen(self, pens, c_poisson):
        for p in pens:
            p.xgreen_peers(self.b[p.rank], c_poisson, self._xgroup(p, self.a))
        self.fence()

    def yinv(self, pens):
        for p in pens:
            p.yinv_peers(self.a[p.rank], self._ygroup(p, self.b))
        self.fence()

    def backward(self, pens):
        for p in pens:
            p.backward_from(self.b[p.rank])


class LocalExchange(_PencilTransposes, _slab.LocalExchange):
    """Every pencil of the decomposition in this process (list index = rank);
    the exchanges are device copies, pencil after pencil."""

    def ghost(self, pens):
        cf = torch.contiguous_format
        rows = [tuple(t.clone(memory_format=cf) for t in (q.xghost(), q.yghost(), q.corner())) for q in pens]
        for q in pens:
            xg = rows[_rank(q, q.rx - 1, q.ry)][0]
            yg = rows[_rank(q, q.rx, q.ry - 1)][1]
            cg = rows[_rank(q, q.rx - 1, q.ry - 1)][2]
            q.fold(xg, yg, cg)

    def ytrans(self, pens, forward: bool):
        for q in pens:
            group = [pens[_rank(q, q.rx, c)] for c in range(q.py)]
            _, rsz = y_splits(q, forward)
            at = 0
            for s, src in enumerate(group):
                ssz, _ = y_splits(src, forward)
                so = sum(ssz[:q.ry])
                q.recv[at:at + rsz[s]].copy_(src.send[so:so + rsz[s]])
                at += rsz[s]

    def xtrans(self, pens):
        for q in pens:
            blk = x_splits(q)[0]
            for s in range(q.px):
                src = pens[_rank(q, s, q.ry)]
                q.recv[s * blk:(s + 1) * blk].copy_(src.send[q.rx * blk:(q.rx + 1) * blk])

    def halo(self, pens):
        for q in pens:  # x rows of the own y range
            nx, ny = q.nx, q.ny
            up, dn = pens[_rank(q, q.rx + 1, q.ry)], pens[_rank(q, q.rx - 1, q.ry)]
            up.halo[0:2, 2:ny + 2].copy_(q.halo[nx:nx + 2, 2:ny + 2])
            dn.halo[nx + 2:nx + 5, 2:ny + 2].copy_(q.halo[2:5, 2:ny + 2])
        for q in pens:  # then y rows over every x row
            ny = q.ny
            up, dn = pens[_rank(q, q.rx, q.ry + 1)], pens[_rank(q, q.rx, q.ry - 1)]
            up.halo[:, 0:2].copy_(q.halo[:, ny:ny + 2])
            dn.halo[:, ny + 2:ny + 5].copy_(q.halo[:, 2:5])


class DistExchange(_PencilTransposes, _slab.DistExchange):
    """This process's one pencil; the transposes are all-to-alls in the row
    and column sub-groups, the ghost rows and halo point-to-point messages.
    Every rank must construct it at the same point (new_group is collective)."""

    def __init__(self, px: int, py: int, group=None):
        super().__init__(group)
        dist = self.dist
        self.px, self.py = px, py
        rank = dist.get_rank(group) if group is not None else dist.get_rank()
        if group is not None:
            members = dist.get_process_group_ranks(group)
        else:
            members = list(range(dist.get_world_size()))
        if len(members) != px * py:
            raise PMError(L.PM_ERR_ARG, f"{len(members)} ranks for a {px} x {py} decomposition")
        self.members = members
        self.ygroups = [dist.new_group([members[rx * py + c] for c in range(py)]) for rx in range(px)]
        self.xgroups = [dist.new_group([members[d * py + ry] for d in range(px)]) for ry in range(py)]
        self.rx, self.ry = rank // py, rank % py

    def _pair(self, q, send_t, to, recv_t, frm):
        """send_t to pencil `to`, recv_t from pencil `frm` (ranks of the
        decomposition); a copy when both are this pencil."""
        if to == q.rank:
            recv_t.copy_(send_t)
        else:
            self._sendrecv(send_t.contiguous(), self.members[to], recv_t, self.members[frm])

    def ghost(self, pens):
        (q,) = pens
        out = []
        for rows, dx, dy in ((q.xghost(), 1, 0), (q.yghost(), 0, 1), (q.corner(), 1, 1)):
            tmp = _empty(rows)
            self._pair(q, rows, _rank(q, q.rx + dx, q.ry + dy), tmp, _rank(q, q.rx - dx, q.ry - dy))
            out.append(tmp)
        q.fold(*out)

    def ytrans(self, pens, forward: bool):
        (q,) = pens
        ssz, rsz = y_splits(q, forward)
        if q.py == 1:
            q.recv[:ssz[0]].copy_(q.send[:ssz[0]])
            return
        self.dist.all_to_all_single(q.recv[:sum(rsz)], q.send[:sum(ssz)], output_split_sizes=rsz,
                                    input_split_sizes=ssz, group=self.ygroups[q.rx])

    def xtrans(self, pens):
        (q,) = pens
        n = sum(x_splits(q))
        if q.px == 1:
            q.recv[:n].copy_(q.send[:n])
            return
        self.dist.all_to_all_single(q.recv[:n], q.send[:n], group=self.xgroups[q.ry])

    def halo(self, pens):
        (q,) = pens
        nx, ny, b = q.nx, q.ny, q.halo
        lo, hi = _empty(b[0:2, 2:ny + 2]), _empty(b[nx + 2:nx + 5, 2:ny + 2])
        self._pair(q, b[nx:nx + 2, 2:ny + 2], _rank(q, q.rx + 1, q.ry), lo, _rank(q, q.rx - 1, q.ry))
        self._pair(q, b[2:5, 2:ny + 2], _rank(q, q.rx - 1, q.ry), hi, _rank(q, q.rx + 1, q.ry))
        b[0:2, 2:ny + 2].copy_(lo)
        b[nx + 2:nx + 5, 2:ny + 2].copy_(hi)
        lo, hi = _empty(b[:, 0:2]), _empty(b[:, ny + 2:ny + 5])
        self._pair(q, b[:, ny:ny + 2], _rank(q, q.rx, q.ry + 1), lo, _rank(q, q.rx, q.ry - 1))
        self._pair(q, b[:, 2:5], _rank(q, q.rx, q.ry - 1), hi, _rank(q, q.rx, q.ry + 1))
        b[:, 0:2].copy_(lo)
        b[:, ny + 2:ny + 5].copy_(hi)


class LocalPeerExchange(_PencilPeerTransposes, LocalExchange):
    """LocalExchange with the transposes done by the kernels' stores into the
    other pencils' buffers (all in one process on one GPU: the pencils' own
    recv / send buffers as A / B; stream order separates the phases)."""

    def __init__(self, pens):
        self.a = [p.recv.data_ptr() for p in pens]
        self.b = [p.send.data_ptr() for p in pens]

    def fence(self):
        pass


class PeerExchange(_PencilPeerTransposes, DistExchange):
    """DistExchange with the four transposes done by the kernels' stores into
    the group members' memory: every rank's own recv / send buffers (A / B)
    mapped into every process by CUDA IPC (slab.PeerBuffers; no multicast),
    a host-side barrier between the phases.  Construct it on every rank at
    the same point (collective)."""

    def __init__(self, pen, px: int, py: int, group=None):
        DistExchange.__init__(self, px, py, group)
        self._peers = _slab.PeerBuffers(pen.lib, self.dist, group, [pen.recv, pen.send])
        self.a, self.b = self._peers.ptrs
        self._stream = pen.stream

    def fence(self):
        self._stream.synchronize()
        self.dist.barrier(group=self.group)

    def close(self):
        self._peers.close()


def step(pens, parts, exchange, mass: float, c_poisson: float, c_kick: float, dt: float):
    """One PM step of a pencil-decomposed mesh.  `pens` / `parts` are every
    pencil of the decomposition (LocalExchange) or this rank's one
    (DistExchange)."""
    step_potential(pens, parts, exchange, mass, c_poisson)
    step_finish(pens, parts, exchange, c_kick, dt)


def step_potential(pens, parts, exchange, mass: float, c_poisson: float):
    """The first part of `step`: deposit, ghost rows, Poisson solve,
    potential halo.  Reads only the particles' cell and offset words (0-3)."""
    for p, q in zip(pens, parts):
        p.deposit(q, mass)
    exchange.ghost(pens)
    exchange.forward(pens)
    exchange.yfwd(pens)
    exchange.xgreen(pens, c_poisson)
    exchange.yinv(pens)
    exchange.backward(pens)
    exchange.halo(pens)


def step_finish(pens, parts, exchange, c_kick: float, dt: float):
    """The rest of `step`: gather + kick + drift, migration."""
    for p, q in zip(pens, parts):
        p.kick_drift(q, c_kick, dt)
    exchange.migrate(pens, parts)


def distribute(cell, off, vel, ids, ng: int, px: int, py: int, ranks, cap_factor: float = 1.5, device=None):
    """SlabParticles for each rank in `ranks`: the particles whose (x, y) cell
    lies in that rank's pencil, with capacity cap_factor x the even share."""
    own = owner_of(cell, ng, px, py)
    share = (cell.numel() + px * py - 1) // (px * py)
    out = []
    for r in ranks:
        sel = torch.nonzero(own == r).flatten()
        q = SlabParticles(max(int(cap_factor * share), sel.numel()) + 64, device if device is not None else cell.device)
        q.set(cell[sel], [a[sel] for a in off], [a[sel] for a in vel], ids[sel])
        out.append(q)
    return out
