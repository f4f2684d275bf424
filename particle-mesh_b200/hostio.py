"""Particle state kept in host memory and stepped on the GPU: the copies of
every step pipelined on two copy streams.

A caller that holds the particles in (pinned) host memory -- the reference's
own model, whose arrays live on the host -- and steps them on the GPU moves
the whole state up and back every step.  PCIe carries the two directions at
once, and the step itself needs the velocities only at its gather, so:

  HostRoundTrip   any step function; the arrays move in particle ranges, a
                  range's upload for the next step waiting only for its own
                  download of this step (serial=True: every copy in order on
                  the compute stream, for comparison)
  SplitRoundTrip  pm_potential_f32 then pm_kick_drift_f32 by ranges (or a
                  decomposed step's potential part, then its gather and
                  migration): the positions go up first, the velocities while
                  the potential is computed, and each range comes down when
                  its gather is done

Every step still copies all of its inputs in and all of its results out;
only the overlap changes.  Events order every copy against the kernels and
the other copies of the same range.
"""
from __future__ import annotations

import torch


class HostRoundTrip:
    """Per step: the particle state from pinned host memory to the device,
    the step, the new state back to the host.  The arrays move in `chunks`
    particle ranges on two copy streams; a chunk's host-to-device copy waits
    for the device-to-host copy of the same range in the previous step (the
    host copy it reads), so every step still moves all of its inputs in and all
    of its results out, and PCIe carries the two directions at once.
    serial=True: every copy on the compute stream, one after another."""

    def __init__(self, stream, dev_arrays, host_arrays, chunks: int = 16, serial: bool = False):
        self.stream, self.dev, self.host = stream, dev_arrays, host_arrays
        self.chunks, self.serial = chunks, serial
        self.h2d = torch.cuda.Stream(device=stream.device)
        self.d2h = torch.cuda.Stream(device=stream.device)
        self.done = []  # (lo, hi, event) of the last step's device-to-host copies

    def _bounds(self, n):
        return [(n * k // self.chunks, n * (k + 1) // self.chunks) for k in range(self.chunks)]

    def start(self, event):
        """Copies of the next step start after `event` (the timing start)."""
        self.h2d.wait_event(event)
        self.d2h.wait_event(event)

    def step(self, n_in: int, run, n_out=None):
        """run() advances the state on the compute stream; n_out() the live
        count after it (particles may migrate); returns (particles copied
        up, particles copied down)."""
        if self.serial:
            with torch.cuda.stream(self.stream):
                for h, d in zip(self.host, self.dev):
                    d[:n_in].copy_(h[:n_in], non_blocking=True)
                run()
                n = n_out() if n_out else n_in
                for h, d in zip(self.host, self.dev):
                    h[:n].copy_(d[:n], non_blocking=True)
            return n_in, n
        arrived = []
        for lo, hi in self._bounds(n_in):
            with torch.cuda.stream(self.h2d):
                for dlo, dhi, ev in self.done:
                    if dlo < hi and lo < dhi:
                        self.h2d.wait_event(ev)
                for h, d in zip(self.host, self.dev):
                    d[lo:hi].copy_(h[lo:hi], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.h2d)
                arrived.append(ev)
        for ev in arrived:
            self.stream.wait_event(ev)
        with torch.cuda.stream(self.stream):
            run()
        n = n_out() if n_out else n_in
        stepped = torch.cuda.Event()
        stepped.record(self.stream)
        self.d2h.wait_event(stepped)
        self.done = []
        for lo, hi in self._bounds(n):
            with torch.cuda.stream(self.d2h):
                for h, d in zip(self.host, self.dev):
                    h[lo:hi].copy_(d[lo:hi], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.d2h)
                self.done.append((lo, hi, ev))
        return n_in, n

    def finish(self):
        """The compute stream waits for the last step's copies (timing end)."""
        for _, _, ev in self.done:
            self.stream.wait_event(ev)


class SplitRoundTrip:
    """HostRoundTrip for a step in two parts: potential(), which reads only the
    first word group (cell, offsets), then kick_drift(range) per particle
    range -- or one finish() for a step that also moves particles between
    ranks.  The first group moves first and the second (velocities, ids)
    after it, in both directions, so the second group's upload runs under the
    potential's kernels and, with kick_drift, each range's download starts
    when its gather is done.  Every step still moves every word of every
    particle in and out; a range of a word group goes up only after its
    download of the step before."""

    def __init__(self, stream, pos_dev, vel_dev, pos_host, vel_host, chunks: int = 16):
        self.stream, self.chunks = stream, chunks
        self.groups = ((pos_dev, pos_host), (vel_dev, vel_host))
        self.h2d = torch.cuda.Stream(device=stream.device)
        self.d2h = torch.cuda.Stream(device=stream.device)
        self.done = None  # [group][range] events of the last downloads

    def start(self, event):
        self.h2d.wait_event(event)
        self.d2h.wait_event(event)

    def _event(self, s):
        ev = torch.cuda.Event()
        ev.record(s)
        return ev

    def step(self, n, potential, kick_drift=None, finish=None, n_out=None):
        """potential() reads the first word group; then either kick_drift(lo,
        hi) per range (downloads follow range by range) or finish() once
        (e.g. gather and particle migration; n_out() gives the live count
        after it).  Returns (particles copied up, particles copied down)."""
        rng = [(n * k // self.chunks, n * (k + 1) // self.chunks) for k in range(self.chunks)]
        up = []
        for g, (dev, host) in enumerate(self.groups):
            evs = []
            for k, (lo, hi) in enumerate(rng):
                with torch.cuda.stream(self.h2d):
                    if self.done is not None:
                        self.h2d.wait_event(self.done[g][k])
                    for h, d in zip(host, dev):
                        d[lo:hi].copy_(h[lo:hi], non_blocking=True)
                    evs.append(self._event(self.h2d))
            up.append(evs)
        for ev in up[0]:
            self.stream.wait_event(ev)
        with torch.cuda.stream(self.stream):
            potential()
        gathered = []
        if finish is None:
            for k, (lo, hi) in enumerate(rng):
                self.stream.wait_event(up[1][k])
                with torch.cuda.stream(self.stream):
                    kick_drift(lo, hi)
                gathered.append(self._event(self.stream))
            n2 = n
        else:
            for ev in up[1]:
                self.stream.wait_event(ev)
            with torch.cuda.stream(self.stream):
                finish()
            n2 = n_out() if n_out else n
            rng = [(n2 * k // self.chunks, n2 * (k + 1) // self.chunks) for k in range(self.chunks)]
            gathered = [self._event(self.stream)] * self.chunks
        self.done = [[], []]
        for g, (dev, host) in enumerate(self.groups):
            for k, (lo, hi) in enumerate(rng):
                with torch.cuda.stream(self.d2h):
                    self.d2h.wait_event(gathered[k])
                    for h, d in zip(host, dev):
                        h[lo:hi].copy_(d[lo:hi], non_blocking=True)
                    self.done[g].append(self._event(self.d2h))
        return n, n2

    def finish(self):
        for evs in self.done or []:
            for ev in evs:
                self.stream.wait_event(ev)
