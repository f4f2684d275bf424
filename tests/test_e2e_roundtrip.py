"""The pipelined host round trips (hostio.HostRoundTrip, SplitRoundTrip; the
bench's end-to-end legs) move the particle state between pinned host memory
and the device every step in particle ranges on two copy streams; a race
between a range's upload and its download of the step before would corrupt
the state without changing the timing.  Here both round trips run several steps from the same state as
plain device stepping (pm_step_f32 on resident arrays), and the host state
they end with must match it: velocities within 1e-6 relative L2, positions
within 1e-5 cells (the deposit's shared-memory atomics sum in no fixed
order).  A range left stale by a race would be off by a whole step.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("mode", ["split", "whole", "serial"])
def test_round_trip_state_matches_resident_steps(pmpkg, mode):
    B = pmpkg.hostio
    ng, nrow, steps, dt = 256, 128, 4, 0.05
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    mass, cp = ng ** 3 / nrow ** 3, 4 * np.pi
    pos, vel = pmpkg.zeldovich_ic(ng, nrow, -1.5, 1.0, seed=11, device="cuda:0")
    plan = pmpkg.Plan(ng, "fp32", "spectral", 4, stream=stream, device=dev)
    cell, off = plan.split(*pos)
    v = [a.float() for a in vel]
    ref = [cell.clone(), *[a.clone() for a in off], *[a.clone() for a in v]]
    for _ in range(steps):
        plan.step_split(ref[0], ref[1:4], ref[4:7], mass, cp, dt, dt)
    dbuf = [cell, *off, *v]
    host = [torch.empty(t.numel(), dtype=t.dtype, pin_memory=True) for t in dbuf]
    for h, d in zip(host, dbuf):
        h.copy_(d)
    for d in dbuf:  # the device copy must come from the host every step
        d.zero_()
    n = cell.numel()
    if mode == "split":
        trip = B.SplitRoundTrip(stream, dbuf[:4], dbuf[4:], host[:4], host[4:])
        for _ in range(steps):
            trip.step(n, lambda: plan.potential_split(cell, off, mass, cp),
                      lambda lo, hi: plan.kick_drift_split(plan.workspace_mesh(), cell[lo:hi],
                                                           [a[lo:hi] for a in off], [a[lo:hi] for a in v], dt, dt))
    else:
        trip = B.HostRoundTrip(stream, dbuf, host, serial=mode == "serial")
        for _ in range(steps):
            trip.step(n, lambda: plan.step_split(cell, off, v, mass, cp, dt, dt))
    trip.finish()
    torch.cuda.synchronize()
    plan.check()
    got = [h.to(dev) for h in host]
    vr, vg = torch.stack(ref[4:7]).double(), torch.stack(got[4:7]).double()
    err = float((vg - vr).norm() / vr.norm())
    assert err < 1e-6, err
    xr, xg = plan.join(ref[0], ref[1:4]), plan.join(got[0], got[1:4])
    d = max(float((torch.remainder(a - b + ng / 2, ng) - ng / 2).abs().max()) for a, b in zip(xg, xr))
    assert d < 1e-5, d
    plan.close()


@pytest.mark.parametrize("decomp", ["slab", "pencil"])
def test_split_round_trip_of_a_decomposed_step(pmpkg, decomp):
    """SplitRoundTrip with finish(): a decomposed step at one rank (its
    potential part, then gather, kick, drift and migration) with the particle
    words copied up and back every step ends with the state of the same
    steps on resident words."""
    ng, nrow, steps, dt = 128, 64, 3, 0.05
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    mass, cp = ng ** 3 / nrow ** 3, 4 * np.pi
    D = getattr(pmpkg, decomp)
    pos, vel = pmpkg.zeldovich_ic(ng, nrow, -1.5, 1.0, seed=13, device="cuda:0")
    plan = pmpkg.Plan(ng, "fp32", "spectral", 4, stream=stream, device=dev)
    cell, off = plan.split(*pos)
    v = [a.float() for a in vel]
    ids = torch.arange(nrow ** 3, dtype=torch.int32, device=dev)

    def make():
        if decomp == "slab":
            dec = D.Slab(ng, 1, 0, "spectral", 4, stream=stream, device=dev)
            (part,) = D.distribute(cell, off, v, ids, ng, 1, [0])
            return dec, part, D.DistExchange()
        dec = D.Pencil(ng, 1, 1, 0, "spectral", 4, stream=stream, device=dev)
        (part,) = D.distribute(cell, off, v, ids, ng, 1, 1, [0])
        return dec, part, D.LocalExchange()

    dec_r, part_r, ex_r = make()
    for _ in range(steps):
        D.step([dec_r], [part_r], ex_r, mass, cp, dt, dt)
    dec, part, ex = make()
    host = torch.empty(part.words.shape, dtype=torch.int32, pin_memory=True)
    host.copy_(part.words)
    part.words.zero_()
    rows_dev = [part.words[w] for w in range(part.words.shape[0])]
    rows_host = [host[w] for w in range(host.shape[0])]
    trip = pmpkg.hostio.SplitRoundTrip(stream, rows_dev[:4], rows_dev[4:], rows_host[:4], rows_host[4:])
    for _ in range(steps):
        trip.step(part.n, lambda: D.step_potential([dec], [part], ex, mass, cp),
                  finish=lambda: D.step_finish([dec], [part], ex, dt, dt), n_out=lambda: part.n)
    trip.finish()
    torch.cuda.synchronize()
    dec.check()
    n = part_r.n
    assert part.n == n
    w, wr = host[:, :n].to(dev), part_r.words[:, :n]
    w, wr = w[:, torch.argsort(w[7])], wr[:, torch.argsort(wr[7])]
    assert torch.equal(w[7], wr[7])
    vg, vr = w[4:7].view(torch.float32).double(), wr[4:7].view(torch.float32).double()
    err = float((vg - vr).norm() / vr.norm())
    assert err < 1e-6, err
    xg = plan.join(w[0].contiguous(), [w[1 + a].view(torch.float32).contiguous() for a in range(3)])
    xr = plan.join(wr[0].contiguous(), [wr[1 + a].view(torch.float32).contiguous() for a in range(3)])
    d = max(float((torch.remainder(a - b + ng / 2, ng) - ng / 2).abs().max()) for a, b in zip(xg, xr))
    assert d < 1e-5, d
    for x in (dec, dec_r):
        x.close()
    plan.close()
