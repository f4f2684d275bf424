"""A CPU stand-in for the per-slab CUDA kernels of the x-slab decomposition.

TEST INFRASTRUCTURE, NOT PRODUCT.  It exposes the same methods and buffers as
``slab.Slab`` (deposit, fold, forward, xgreen, backward, kick_drift and the
migration sort / pack / unpack, with the same buffer layouts) computed in FP64
with numpy, so that the exchange logic of ``slab.step`` / ``slab.DistExchange``
can run on gloo ranks on CPU.  The CUDA path never imports this module.

Semantics follow the kernels:
  buffer planes [nx + 6][ng][ng + 2]: 0-1 lower halo, 2..nx+1 own planes,
  nx+2 the ghost plane / upper halo; spectra are H = ng/2 + 1 complex per row;
  transposes pack rows [ky][x] (forward), [kyl][kx] (x pass), [x owner][kyl][x]
  (back); CIC deposit without a half-cell shift (include/utils/utils_inline.h
  :25-49), 4-point centred gradient fused into the trilinear gather.
"""
from __future__ import annotations

import numpy as np
import torch

WORDS = 8


def split1(v: np.ndarray, ng: int):
    f = np.floor(v)
    cell = np.mod(f.astype(np.int64), ng)
    off = (v - f).astype(np.float32)
    up = off >= 1.0
    off[up] = 0.0
    cell[up] = (cell[up] + 1) % ng
    return cell, off


def pack_cell(i, j, k):
    return ((i.astype(np.int64) << 20) | (j.astype(np.int64) << 10) | k.astype(np.int64)).astype(np.uint32)


def unpack_cell(c):
    c = np.asarray(c).astype(np.uint32).astype(np.int64)
    return c >> 20, (c >> 10) & 1023, c & 1023


class CpuSlab:
    def __init__(self, ng: int, nranks: int, rank: int, green: str = "spectral", grad_order: int = 4):
        assert green == "spectral" and grad_order == 4
        self.ng, self.nranks, self.rank = ng, nranks, rank
        self.nx = ng // nranks
        self.x0 = rank * self.nx
        self.h = ng // 2 + 1
        self.buf = torch.zeros((self.nx + 6, ng, ng + 2), dtype=torch.float64)
        self.send = torch.zeros(self.nx * ng * (ng + 2), dtype=torch.float64)
        self.recv = torch.zeros_like(self.send)
        self._perm = None

    def ghost_plane(self):
        return self.buf[self.nx + 2]

    def potential(self):
        return self.buf[2:self.nx + 2]

    def check(self):
        pass

    def _spec(self, t, shape):
        return t.numpy().view(np.complex128).reshape(shape)

    # ---- deposit + z R2C (own planes background -1, ghost plane 0)
    def deposit(self, q, mass):
        ng, nx = self.ng, self.nx
        n = q.n
        w = q.words[:, :n].numpy()
        i, j, k = unpack_cell(w[0].view(np.uint32))
        off = [w[1 + a].view(np.float32).astype(np.float64) for a in range(3)]
        li = i - self.x0
        assert np.all((li >= 0) & (li < nx)), "particle outside its slab"
        rho = np.zeros((nx + 1, ng, ng))
        for a in (0, 1):
            wa = off[0] if a else 1.0 - off[0]
            for b in (0, 1):
                wb = off[1] if b else 1.0 - off[1]
                for c in (0, 1):
                    wc = off[2] if c else 1.0 - off[2]
                    np.add.at(rho, (li + a, (j + b) % ng, (k + c) % ng), mass * wa * wb * wc)
        rho[:nx] -= 1.0
        b = self.buf.numpy()
        b[2:nx + 6] = 0.0
        spec = np.fft.rfft(rho, axis=2)
        b[2:nx + 3].view(np.complex128)[:] = spec

    def fold(self, ghost):
        self.buf[2] += ghost

    def _yfwd_rows(self):
        """y forward of the own planes, as rows [ky][x][kz]."""
        nx = self.nx
        own = self.buf[2:nx + 2].numpy().view(np.complex128)
        own[:] = np.fft.fft(own, axis=1)
        return own.transpose(1, 0, 2)

    def forward(self):
        ng, nx, h = self.ng, self.nx, self.h
        self._spec(self.send, (ng, nx, h))[:] = self._yfwd_rows()

    def forward_peers(self, peer_recv):
        """The rows of ky in rank d's range stored into peer_recv[d], block
        `rank` (the layout the all-to-all would deliver)."""
        nx, h, p = self.nx, self.h, self.nranks
        rows = self._yfwd_rows()
        for d in range(p):
            self._spec(peer_recv[d], (p, nx, nx, h))[self.rank] = rows[d * nx:(d + 1) * nx]

    def xgreen(self, c_poisson):
        ng, nx, h, p = self.ng, self.nx, self.h, self.nranks
        self._spec(self.send, (p, nx, nx, h))[:] = self._xgreen_lines(self.recv, c_poisson).reshape(
            nx, p, nx, h).transpose(1, 0, 2, 3)

    def xgreen_peers(self, recv, c_poisson, peer_rows):
        """x + Green on `recv`; line element kx stored into peer_rows[kx // nx]
        as row (ky0 + kyl, kx mod nx), i.e. its block `rank`."""
        nx, h, p = self.nx, self.h, self.nranks
        x = self._xgreen_lines(recv, c_poisson)
        for d in range(p):
            self._spec(peer_rows[d], (p, nx, nx, h))[self.rank] = x[:, d * nx:(d + 1) * nx]

    def _xgreen_lines(self, recv, c_poisson):
        ng, nx, h, p = self.ng, self.nx, self.h, self.nranks
        nyl = nx
        r = self._spec(recv, (p, nyl, nx, h))
        x = r.transpose(1, 0, 2, 3).reshape(nyl, ng, h)
        x = np.fft.fft(x, axis=1)
        kx = np.arange(ng)[None, :, None]
        ky = (self.x0 + np.arange(nyl))[:, None, None]
        kz = np.arange(h)[None, None, :]
        mx, my = np.where(kx <= ng // 2, kx, kx - ng), np.where(ky <= ng // 2, ky, ky - ng)
        w = 2.0 * np.pi / ng
        with np.errstate(divide="ignore", invalid="ignore"):
            g = -c_poisson / (float(ng) ** 3 * w * w * (mx * mx + my * my + kz * kz))
        g[(mx == 0) & (my == 0) & (kz == 0)] = 0.0
        return np.fft.ifft(x * g, axis=1) * ng

    def backward(self):
        self.backward_rows(self.recv)

    def backward_rows(self, rows):
        ng, nx, h = self.ng, self.nx, self.h
        spec = self._spec(rows, (ng, nx, h)).transpose(1, 0, 2)
        spec = np.fft.ifft(spec, axis=1) * ng
        phi = np.fft.irfft(spec, n=ng, axis=2) * ng
        b = self.buf.numpy()
        b[2:nx + 2, :, :ng] = phi
        b[2:nx + 2, :, ng:] = 0.0

    # ---- fused 4-point gradient + trilinear gather, kick, drift
    def kick_drift(self, q, c_kick, dt):
        ng = self.ng
        n = q.n
        w = q.words[:, :n].numpy()
        i, j, k = unpack_cell(w[0].view(np.uint32))
        off = [w[1 + a].view(np.float32).astype(np.float64) for a in range(3)]
        vel = [w[4 + a].view(np.float32) for a in range(3)]
        li = i - self.x0
        assert np.all((li >= 0) & (li < self.nx))
        phi = self.buf.numpy()

        def P(dx, dy, dz):
            return phi[li + 2 + dx, (j + dy) % ng, (k + dz) % ng]

        def D(f, s):  # minus the 4-point centred derivative at offset s along one axis
            return (8.0 * (f(s - 1) - f(s + 1)) - (f(s - 2) - f(s + 2))) / 12.0

        g = [np.zeros(n) for _ in range(3)]
        for a in (0, 1):
            wa = off[0] if a else 1.0 - off[0]
            for b in (0, 1):
                wb = off[1] if b else 1.0 - off[1]
                for c in (0, 1):
                    wc = off[2] if c else 1.0 - off[2]
                    wt = wa * wb * wc
                    g[0] += wt * D(lambda s: P(s, b, c), a)
                    g[1] += wt * D(lambda s: P(a, s, c), b)
                    g[2] += wt * D(lambda s: P(a, b, s), c)
        u = [vel[a].astype(np.float64) + c_kick * g[a] for a in range(3)]
        for a in range(3):
            w[4 + a].view(np.float32)[:] = u[a].astype(np.float32)
        if dt != 0.0:
            u32 = [w[4 + a].view(np.float32).astype(np.float64) for a in range(3)]
            pos = [(i, j, k)[a] + off[a] + u32[a] * dt for a in range(3)]
            cells, offs = zip(*(split1(np.mod(pp, ng), ng) for pp in pos))
            w[0].view(np.uint32)[:] = pack_cell(*cells)
            for a in range(3):
                w[1 + a].view(np.float32)[:] = offs[a]

    # ---- migration
    def migrate_sort(self, q):
        c = q.words[0, :q.n].numpy().view(np.uint32).astype(np.int64)
        own = ((c >> 20) % self.ng) // self.nx
        self._perm = np.argsort(own, kind="stable")
        return [int(v) for v in np.bincount(own, minlength=self.nranks)]

    def migrate_pack(self, q, packed):
        packed[:q.n] = q.words[:, torch.from_numpy(self._perm)].T

    def migrate_unpack(self, packed, n, q, at):
        assert at + n <= q.cap
        q.words[:, at:at + n] = packed[:n].T
