"""A CPU stand-in for the per-pencil CUDA kernels of the pencil decomposition.

TEST INFRASTRUCTURE, NOT PRODUCT.  It exposes the same methods and buffers as
``pencil.Pencil`` (deposit, fold, forward, yfwd, xgreen, yinv, backward,
kick_drift, the migration sort / pack / unpack), computed in FP64 with numpy
on the kernels' buffer layouts, so that the exchange logic of ``pencil.step``
and ``pencil.DistExchange`` can run on gloo ranks on CPU.  The CUDA path never
imports this module.

Layouts (complex = 2 floats, h = ng/2 + 1, kz chunk c = [kb(c), kb(c+1))):
  halo [nx + 5][ny + 5][ng + 2]  row (x - x0 + 2, y - y0 + 2)
  forward send   chunk c as [nx][ny][hc(c)] at complex offset nx ny kb(c)
  yfwd send      ky chunk d as [nx][nx][hc] at block d
  xgreen         recv [px][nx][nx][hc] = x lines [ng][nx][hc]; send = recv
  yinv send      y block d as [nx][ny][hc] at block d
  backward recv  from member s: [nx][ny][hc(s)] at complex offset nx ny kb(s)
"""
from __future__ import annotations

import numpy as np
import torch

from slab_cpu import pack_cell, split1, unpack_cell


class CpuPencil:
    def __init__(self, ng: int, px: int, py: int, rank: int, green: str = "spectral", grad_order: int = 4):
        assert green == "spectral" and grad_order == 4
        self.ng, self.px, self.py, self.rank = ng, px, py, rank
        self.nranks, self.rx, self.ry = px * py, rank // py, rank % py
        self.nx, self.ny, self.h = ng // px, ng // py, ng // 2 + 1
        self.x0, self.y0 = self.rx * self.nx, self.ry * self.ny
        hcmax = -(-self.h // py)
        self.halo = torch.zeros((self.nx + 5, self.ny + 5, ng + 2), dtype=torch.float64)
        self.send = torch.zeros(2 * self.nx * ng * hcmax, dtype=torch.float64)
        self.recv = torch.zeros_like(self.send)
        self._perm = None

    def kb(self, c):
        return (c * self.h) // self.py

    def hc(self, c):
        return self.kb(c + 1) - self.kb(c)

    def _c(self, t, off, shape):  # complex view of floats [2 off, ...)
        n = int(np.prod(shape))
        return t.numpy()[2 * off:2 * (off + n)].view(np.complex128).reshape(shape)

    def xghost(self):
        return self.halo[self.nx + 2, 2:self.ny + 2]

    def yghost(self):
        return self.halo[2:self.nx + 2, self.ny + 2]

    def corner(self):
        return self.halo[self.nx + 2, self.ny + 2:self.ny + 3]

    def potential(self):
        return self.halo[2:self.nx + 2, 2:self.ny + 2]

    def check(self):
        pass

    def deposit(self, q, mass):
        ng, nx, ny = self.ng, self.nx, self.ny
        w = q.words[:, :q.n].numpy()
        i, j, k = unpack_cell(w[0].view(np.uint32))
        off = [w[1 + a].view(np.float32).astype(np.float64) for a in range(3)]
        li, lj = i - self.x0, j - self.y0
        assert np.all((li >= 0) & (li < nx) & (lj >= 0) & (lj < ny)), "particle outside its pencil"
        b = self.halo.numpy()
        b[:] = 0.0
        b[2:nx + 2, 2:ny + 2, :ng] = -1.0
        for a in (0, 1):
            wa = off[0] if a else 1.0 - off[0]
            for bb in (0, 1):
                wb = off[1] if bb else 1.0 - off[1]
                for c in (0, 1):
                    wc = off[2] if c else 1.0 - off[2]
                    np.add.at(b, (li + 2 + a, lj + 2 + bb, (k + c) % ng), mass * wa * wb * wc)

    def fold(self, xg, yg, corner):
        self.halo[2, 2:self.ny + 2] += xg
        self.halo[2:self.nx + 2, 2] += yg
        self.halo[2, 2] += corner[0]

    def _zfwd(self):
        nx, ny, ng = self.nx, self.ny, self.ng
        self._own = np.fft.rfft(self.halo.numpy()[2:nx + 2, 2:ny + 2, :ng], axis=2)

    def forward(self):
        nx, ny = self.nx, self.ny
        self._zfwd()
        for c in range(self.py):
            self._c(self.send, nx * ny * self.kb(c), (nx, ny, self.hc(c)))[:] = \
                self._own[:, :, self.kb(c):self.kb(c + 1)]

    def forward_peers(self, peer_a):
        """kz chunk c into peer_a[c] (y member c), block ry."""
        nx, ny = self.nx, self.ny
        self._zfwd()
        for c in range(self.py):
            self._c(peer_a[c], self.ry * nx * ny * self.hc(c), (nx, ny, self.hc(c)))[:] = \
                self._own[:, :, self.kb(c):self.kb(c + 1)]

    def _ywork(self, inp):
        nx, ny, ng, hc = self.nx, self.ny, self.ng, self.hc(self.ry)
        r = self._c(inp, 0, (self.py, nx, ny, hc))
        return np.fft.fft(r.transpose(1, 0, 2, 3).reshape(nx, ng, hc), axis=1)

    def yfwd(self):
        nx, hc = self.nx, self.hc(self.ry)
        work = self._ywork(self.recv)
        self._c(self.send, 0, (self.px, nx, nx, hc))[:] = work.reshape(nx, self.px, nx, hc).transpose(1, 0, 2, 3)

    def yfwd_peers(self, inp, peer_b):
        """ky chunk d into peer_b[d] (x member d), block rx."""
        nx, hc = self.nx, self.hc(self.ry)
        work = self._ywork(inp)
        for d in range(self.px):
            self._c(peer_b[d], self.rx * nx * nx * hc, (nx, nx, hc))[:] = work[:, d * nx:(d + 1) * nx]

    def xgreen(self, c_poisson):
        nx, ng, hc = self.nx, self.ng, self.hc(self.ry)
        self._c(self.send, 0, (ng, nx, hc))[:] = self._xlines(self.recv, c_poisson)

    def xgreen_peers(self, inp, c_poisson, peer_a):
        """x block d into peer_a[d] (x member d), block rx."""
        nx, hc = self.nx, self.hc(self.ry)
        x = self._xlines(inp, c_poisson)
        for d in range(self.px):
            self._c(peer_a[d], self.rx * nx * nx * hc, (nx, nx, hc))[:] = x[d * nx:(d + 1) * nx]

    def _xlines(self, inp, c_poisson):
        nx, ng, hc = self.nx, self.ng, self.hc(self.ry)
        x = np.fft.fft(self._c(inp, 0, (ng, nx, hc)), axis=0)
        kx = np.arange(ng)[:, None, None]
        ky = (self.rx * nx + np.arange(nx))[None, :, None]
        kz = (self.kb(self.ry) + np.arange(hc))[None, None, :]
        mx, my = np.where(kx <= ng // 2, kx, kx - ng), np.where(ky <= ng // 2, ky, ky - ng)
        w = 2.0 * np.pi / ng
        with np.errstate(divide="ignore", invalid="ignore"):
            g = -c_poisson / (float(ng) ** 3 * w * w * (mx * mx + my * my + kz * kz))
        g[(mx == 0) & (my == 0) & (kz == 0)] = 0.0
        return np.fft.ifft(x * g, axis=0) * ng

    def _yiwork(self, inp):
        nx, ng, hc = self.nx, self.ng, self.hc(self.ry)
        r = self._c(inp, 0, (self.px, nx, nx, hc))
        return np.fft.ifft(r.transpose(1, 0, 2, 3).reshape(nx, ng, hc), axis=1) * ng

    def yinv(self):
        nx, ny, hc = self.nx, self.ny, self.hc(self.ry)
        work = self._yiwork(self.recv)
        self._c(self.send, 0, (self.py, nx, ny, hc))[:] = work.reshape(nx, self.py, ny, hc).transpose(1, 0, 2, 3)

    def yinv_peers(self, inp, peer_b):
        """y block d into peer_b[d] (y member d), at its kz chunk ry."""
        nx, ny, hc = self.nx, self.ny, self.hc(self.ry)
        work = self._yiwork(inp)
        for d in range(self.py):
            self._c(peer_b[d], nx * ny * self.kb(self.ry), (nx, ny, hc))[:] = work[:, d * ny:(d + 1) * ny]

    def backward(self):
        self.backward_from(self.recv)

    def backward_from(self, inp):
        nx, ny, ng = self.nx, self.ny, self.ng
        own = np.empty((nx, ny, self.h), dtype=np.complex128)
        for s in range(self.py):
            own[:, :, self.kb(s):self.kb(s + 1)] = self._c(inp, nx * ny * self.kb(s), (nx, ny, self.hc(s)))
        b = self.halo.numpy()
        b[2:nx + 2, 2:ny + 2, :ng] = np.fft.irfft(own, n=ng, axis=2) * ng
        b[2:nx + 2, 2:ny + 2, ng:] = 0.0

    def kick_drift(self, q, c_kick, dt):
        ng = self.ng
        n = q.n
        w = q.words[:, :n].numpy()
        i, j, k = unpack_cell(w[0].view(np.uint32))
        off = [w[1 + a].view(np.float32).astype(np.float64) for a in range(3)]
        vel = [w[4 + a].view(np.float32) for a in range(3)]
        li, lj = i - self.x0, j - self.y0
        assert np.all((li >= 0) & (li < self.nx) & (lj >= 0) & (lj < self.ny))
        phi = self.halo.numpy()

        def P(dx, dy, dz):
            return phi[li + 2 + dx, lj + 2 + dy, (k + dz) % ng]

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

    def migrate_sort(self, q):
        c = q.words[0, :q.n].numpy().view(np.uint32).astype(np.int64)
        own = (((c >> 20) % self.ng) // self.nx) * self.py + (((c >> 10) & 1023) % self.ng) // self.ny
        self._perm = np.argsort(own, kind="stable")
        return [int(v) for v in np.bincount(own, minlength=self.nranks)]

    def migrate_pack(self, q, packed):
        packed[:q.n] = q.words[:, torch.from_numpy(self._perm)].T

    def migrate_unpack(self, packed, n, q, at):
        assert at + n <= q.cap
        q.words[:, at:at + n] = packed[:n].T
