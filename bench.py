#!/usr/bin/env python
"""Throughput of the particle-mesh step on B200: particle-updates/s.

Workload (default): 512^3 particles on a 1024^3 periodic mesh, Zel'dovich
initial conditions (P(k) ~ k^-1.5, rms displacement 1.0 cell, seeded,
synthetic), spectral Poisson, 4-point gradient, leapfrog step of dt = 0.005.
One step = deposit, Poisson solve, gradient + interpolation + kick + drift
over every particle; particle-updates/s = particles x steps / time.

  value      the FP32 split-position path (the fast path), inputs resident in
             HBM, K steps timed with CUDA events (max over ranks)
  fp64       the plain FP64 path on the same initial state
  force_err  relative L2 of FP32 vs FP64 particle forces on that state
  e2e        the FP32 step through the C ABI (pm_potential_f32, then
             pm_kick_drift_f32 over particle ranges) with the particle state
             copied from pinned host memory and back every step, on two copy
             streams so both PCIe directions and the kernels overlap; the
             whole-step and serial figures beside it
  roofline   dominant kernel, algorithmic bytes / CUDA-event time, vs the
             measured HBM copy bandwidth
  cpu_baseline the reference's CPU code on a bounded sample (rank 0, N = 1)
  fp64_256   the FP64 path on 256^3 particles / 256^3 mesh, 20 KDK steps
  accuracy   FP32 vs FP64 after the configuration's 50 KDK steps (positions,
             velocities, density) and FP64-summed mass / momentum drift
  adjoint    adjoint step vs forward step at 128^3 (FP32 split path; FP64 check
             path under "fp64")

Multi-GPU (torchrun): the configuration's one box is split into x-slabs, one
per GPU (strong scaling; NCCL ghost fold, spectrum transposes, potential halo
and particle migration every step), and the ensemble's boxes are dealt to the
GPUs; every timing is the max over ranks.  --pencil splits it into px x py
pencils instead (x and y; two sub-group transposes).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "particle-mesh_b200"))

METRIC = "PM particle-updates/s, 512^3 on 1024^3 mesh: FP32 vs FP64 at force err <=1e-4"
UNIT = "particle-updates/s"
N_S, RMS, DT, SEED = -1.5, 1.0, 0.005, 1000
CPU_SAMPLE = (256, 128)  # (mesh, particles per side): 1/64 of the workload
ACC_STEPS = 50  # the mixed-precision configuration's run length
# the ensemble autotuner's choices for B200, committed (pm_ensemble_create
# reads it and measures only the shapes it lacks)
TUNE_CACHE = os.path.join(ROOT, "particle-mesh_b200", "tune_b200.txt")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ng", type=int, default=1024)
    ap.add_argument("--nrow", type=int, default=512)
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-ensemble", action="store_true")
    ap.add_argument("--skip-adjoint", action="store_true")
    ap.add_argument("--skip-accuracy", action="store_true")
    ap.add_argument("--ensemble-boxes", type=int, default=256)
    ap.add_argument("--gather", default="cached", choices=["cached", "tiled"],
                    help="gather of the FP32 step (pm_plan_set_gather)")
    ap.add_argument("--slab", action="store_true",
                    help="run the x-slab decomposition at N = 1 too (at N > 1 it is the default)")
    ap.add_argument("--peer", action="store_true",
                    help="slab path: the transposes by the FFT kernels' stores into the other GPUs' memory "
                         "(symmetric memory) instead of NCCL all-to-alls")
    ap.add_argument("--pencil", action="store_true",
                    help="run the pencil decomposition instead (px x py = N pencils, px >= py; 1 x 1 at N = 1)")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples every 100 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id=None):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"]
        if bus_id:
            cmd += ["-i", bus_id]
        try:
            self.p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in out.strip().splitlines():
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def bus_id(torch, dev):
    try:
        p = torch.cuda.get_device_properties(dev)
        return f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
    except Exception:  # noqa: BLE001
        return None


# ------------------------------------------------------- ranks and timing
def reduce_max(v: float, world: int, device=None) -> float:
    """Max of a per-rank time over all ranks (every rank takes this step)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def throughput(world: int, particles_per_rank: int, steps: int, t_ms: float) -> float:
    """Whole-job particle-updates/s: every rank advances its own box."""
    return world * particles_per_rank * steps / (t_ms / 1e3)


def rank_seed(rank: int) -> int:
    """Each rank's box has its own initial conditions."""
    return SEED + rank


# ------------------------------------------------------------- byte model
def stage_bytes(stage: str, ng: int, np_: int, esz: int) -> float:
    """Algorithmic bytes of one launch of a stage (the minimum it must move).

    mesh passes read and write the padded mesh once; particle stages read
    (and write) their particle arrays once and read each mesh cell once."""
    mesh = ng * ng * (ng + 2) * esz
    cells = ng ** 3
    if stage == "mesh_init":
        return mesh
    if stage.startswith("fft_") or stage == "green":
        return 2.0 * mesh
    if esz == 4:  # split positions: cell 4 + offsets 12 (+ velocity 12)
        # bin: cells read twice, permutation written; deposit: permutation +
        # cell + offsets read, every mesh cell written once
        return {"bin": 12 * np_, "deposit": 20 * np_ + mesh, "kick_drift": 56 * np_ + cells * 4,
                "interp": 16 * np_ + 12 * np_ + cells * 4, "sort": 64 * np_}.get(stage, 0.0)
    return {"deposit": 24 * np_ + 2 * mesh, "gradient": mesh + 3 * cells * 8,
            "interp_kick": 72 * np_ + 3 * cells * 8, "drift": 72 * np_}.get(stage, 0.0)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


def ncu_traffic(stage: str, ng: int):
    """DRAM bytes per launch of a stage from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            j = json.load(f)
        e = j.get(f"{stage}@{ng}")
        return float(e["dram_bytes_per_launch"]) if e else None
    except Exception:  # noqa: BLE001
        return None


# -------------------------------------------------------------- CPU side
def cpu_reference_steps(steps: int, warmup: int, budget_s: float | None = None):
    """The reference's CPU step (its own compiled kernels from oracle/_ref,
    scipy.fft with all cores standing in for FFTW) plus a drift, on the
    bounded sample: 128^3 particles on a 256^3 periodic mesh with the same
    initial-condition recipe -- 1/64 of the workload, one rank's share of a
    64-rank run.  OpenMP threads and FFT workers use every host core.
    Returns (particle-updates/s, threads, seconds)."""
    import numpy as np
    import scipy.fft
    from oracle import oracle as O

    ng, nrow = CPU_SAMPLE
    R = O.ref_lib()
    kind = "reference" if R is not None else "port"
    cores = len(os.sched_getaffinity(0))
    pos, vel = O.zeldovich_ic(ng, nrow, N_S, RMS, SEED)
    x, y, z = (np.ascontiguousarray(a) for a in pos)
    v = [np.ascontiguousarray(a) for a in vel]
    mass = ng ** 3 / nrow ** 3
    a_ref = O.START_A
    rfftn = lambda a, **k: scipy.fft.rfftn(a, workers=cores, **k)  # noqa: E731
    irfftn = lambda a, **k: scipy.fft.irfftn(a, workers=cores, **k)  # noqa: E731
    steppers = {}

    def one(threads):
        t0 = time.perf_counter()
        if R is not None:
            if threads not in steppers:
                steppers[threads] = O.ReferenceStepper(ng, a_ref, threads, rfftn, irfftn)
                steppers[threads].keep = False
            steppers[threads].step(x, y, z, *v, mass)
        else:
            cp, ck = O.reference_coefficients(a_ref)
            O.force_step(ng, x, y, z, *v, mass, cp, ck, fft="numpy")
        O.drift(ng, x, y, z, *v, DT)
        return time.perf_counter() - t0

    try:
        # every host core: OpenMP threads for the reference kernels, workers
        # for the FFT (the restated port, without the reference, is serial)
        best = cores if R is not None else 1
        for _ in range(max(1, warmup)):  # the first call pays the setup
            one(best)
        ts = []
        t_start = time.perf_counter()
        for _ in range(steps):
            ts.append(one(best))
            if budget_s and time.perf_counter() - t_start > budget_s:
                break
        stage_s = None
        if R is not None:
            st = steppers[best]
            stage_s = dict(st.timers)
    finally:
        for st in steppers.values():
            st.close()
    t = sum(ts) / len(ts)
    per_step = {k: v / (len(ts) + max(1, warmup)) for k, v in (stage_s or {}).items()}
    return {"value": nrow ** 3 / t, "omp_threads": best, "cores": cores, "seconds": t, "steps": len(ts),
            "kind": kind, "stage_s_approx": per_step}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    steps = max(1, args.steps)
    r = cpu_reference_steps(steps, args.warmup)
    val, t, n, kind = r["value"], r["seconds"], r["steps"], r["kind"]
    ng, nrow = CPU_SAMPLE
    sample = (f"{nrow}^3 particles on a {ng}^3 periodic mesh (1/64 of the workload: one rank's share of a "
              f"64-rank run), same Zel'dovich recipe; reference kernels from oracle/_ref, scipy.fft for FFTW")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
            "steps": n, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.nrow}^3 particles on {args.ng}^3 mesh, sampled on the CPU as {sample}"},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": r["cores"], "omp_threads": r["omp_threads"],
                             "kind": kind, "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------- ensemble
def ensemble_leg(pm, torch, args, world, rank, dev, stream, barrier, max_over_ranks):
    """The batched-ensemble configuration: 256 boxes with mesh sizes drawn
    from {32, 48, 64, 96, 128}, 20 KDK steps as one CUDA graph.  The box list
    is the same on every rank; at N GPUs the boxes are dealt to the ranks
    (largest first to the least loaded; independent boxes, no collective) and
    the throughput counts every box over the slowest rank's time."""
    import numpy as np
    nb_ = args.ensemble_boxes
    rng = np.random.default_rng(4242)
    sizes = [int(v) for v in rng.choice([32, 48, 64, 96, 128], nb_)]
    n_s = rng.uniform(-2.5, -1.0, nb_)
    rms = rng.uniform(0.2, 1.0, nb_)
    mine = pm.slab.deal_boxes([n ** 3 for n in sizes], world)[rank]
    cells_, offs_, vels_ = [], [[], [], []], [[], [], []]
    for b in mine:
        ngb = sizes[b]
        pb, vb_ = pm.zeldovich_ic(ngb, ngb, float(n_s[b]), float(rms[b]), 100000 + b, device=dev)
        splitter = pm.Plan(ngb, "fp32", "spectral", 4, stream=stream, device=dev)
        cb, ob = splitter.split(*pb)
        cells_.append(cb)
        for a in range(3):
            offs_[a].append(ob[a])
            vels_[a].append(vb_[a].float())
        splitter.close()
        del pb, vb_
    ecell = torch.cat(cells_)
    eoff = [torch.cat(t) for t in offs_]
    evel = [torch.cat(t) for t in vels_]
    del cells_, offs_, vels_
    enp = [sizes[b] ** 3 for b in mine]
    t0 = time.perf_counter()
    ens = pm.Ensemble([sizes[b] for b in mine], enp, [1.0] * len(mine), "spectral", 4, autotune=True,
                      tune_cache=TUNE_CACHE if os.path.exists(TUNE_CACHE) else None)
    t_setup = time.perf_counter() - t0
    cp = pm.unit_box_coefficients(0.01)[0]
    esteps, edt = 20, 0.01
    init = (ecell.clone(), [t.clone() for t in eoff], [t.clone() for t in evel])

    def restore():
        """The configuration's initial state into the graph's particle arrays."""
        ecell.copy_(init[0])
        for a in range(3):
            eoff[a].copy_(init[1][a])
            evel[a].copy_(init[2][a])

    ens.run(ecell, eoff, evel, cp, edt, esteps)  # capture + first replay
    torch.cuda.synchronize()
    reps = 3
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    runs = []
    for _ in range(reps):  # each timed run: the 20 KDK steps from the initial state
        restore()
        torch.cuda.synchronize()
        barrier()
        e0.record(stream)
        ens.run(ecell, eoff, evel, cp, edt, esteps)
        e1.record(stream)
        torch.cuda.synchronize()
        runs.append(e0.elapsed_time(e1))
    barrier()
    t_ens = max_over_ranks(sum(runs)) / reps
    # one more run continuing from the state those steps reached (steps 21 - 40)
    torch.cuda.synchronize()
    e0.record(stream)
    ens.run(ecell, eoff, evel, cp, edt, esteps)
    e1.record(stream)
    torch.cuda.synchronize()
    t_cont = max_over_ranks(e0.elapsed_time(e1))
    # the same run launched eagerly (no graph): the launch overhead the graph removes
    ec, eo, ev = init[0].clone(), [t.clone() for t in init[1]], [t.clone() for t in init[2]]
    torch.cuda.synchronize()
    e0.record(stream)
    for s_ in range(esteps + 1):
        ens.step(ec, eo, ev, cp, (0.5 if s_ in (0, esteps) else 1.0) * edt, edt if s_ < esteps else 0.0)
    e1.record(stream)
    torch.cuda.synchronize()
    t_eager = max_over_ranks(e0.elapsed_time(e1))
    del ec, eo, ev
    info = ens.info()
    total = int(sum(n ** 3 for n in sizes))
    out = {"config": f"{nb_} boxes, mesh sizes drawn from {{32,48,64,96,128}}, particles = cells, "
                     f"P(k)~k^n n~U[-2.5,-1], rms~U[0.2,1.0] cell, {esteps} KDK steps dt={edt}, FP32 split",
           "particles": total, "value": total * esteps / (t_ens / 1e3),
           "unit": UNIT, "ms_per_run": t_ens, "ms_per_step": t_ens / esteps,
           "boxes_per_rank": len(mine), "graph_nodes": info["graph_nodes"], "classes": info["classes"],
           "continued_ms_per_run": t_cont,
           "eager_ms_per_run": t_eager,
           "launch_overhead_removed_by_graph": {"ms_per_run": t_eager - t_ens,
                                                "share_of_eager": (t_eager - t_ens) / t_eager,
                                                "us_per_node": (t_eager - t_ens) * 1e3 / max(1, info["graph_nodes"])},
           "tune_cache": "committed" if os.path.exists(TUNE_CACHE) else "autotuned at creation",
           "setup_s_incl_autotune": t_setup,
           "note": "one CUDA graph per run of 20 KDK steps (21 force evaluations); batched kernels per "
                   "mesh-size class, classes on parallel graph branches; boxes dealt to ranks; every timed run "
                   "starts from the initial conditions (the state copied back outside the timed region); "
                   "continued_ms_per_run: steps 21-40 from the state the timed runs reached"}
    ens.close()
    del ens, ecell, eoff, evel, init
    torch.cuda.empty_cache()
    return out


def pencil_grid(world: int):
    """px x py = world, px the larger power-of-two factor."""
    px = 1
    while px * px < world:
        px *= 2
    return px, world // px


# --------------------------------------------------- N GPUs: one slab each
def ours_slab(args, pm, torch, dist, world, rank, dev, stream, barrier, max_over_ranks):
    """The configuration's one box (512^3 particles on a 1024^3 mesh) split
    over the N GPUs as x-slabs (strong scaling): per step the ghost-plane
    fold, two all-to-all transposes of the spectrum, the potential halo and
    the particle migration go over NCCL (slab.DistExchange).  With --pencil,
    px x py pencils (pencil.DistExchange: row / column sub-groups)."""
    S = pm.slab
    P = pm.pencil
    px, py = pencil_grid(world)
    ng, nrow = args.ng, args.nrow
    np_ = nrow ** 3
    mass = ng ** 3 / np_
    cp, ck = pm.unit_box_coefficients(DT)
    pos, vel = pm.zeldovich_ic(ng, nrow, N_S, RMS, rank_seed(0), device=dev)  # the one box, on every rank
    splitter = pm.Plan(ng, "fp32", "spectral", 4, stream=stream, device=dev)
    cell, off = splitter.split(*pos)
    splitter.close()
    v32 = [a.float() for a in vel]
    ids = torch.arange(np_, dtype=torch.int32, device=dev)
    del pos, vel
    if args.pencil:
        (part,) = P.distribute(cell, off, v32, ids, ng, px, py, [rank])
    else:
        (part,) = S.distribute(cell, off, v32, ids, ng, world, [rank])
    del cell, off, v32, ids
    torch.cuda.empty_cache()
    if args.pencil:
        slab = P.Pencil(ng, px, py, rank, "spectral", 4, stream=stream, device=dev)
        if args.peer:
            ex = P.PeerExchange(slab, px, py) if world > 1 else P.LocalPeerExchange([slab])
        else:
            ex = P.DistExchange(px, py) if world > 1 else P.LocalExchange()
        step_fn = P.step
    else:
        slab = S.Slab(ng, world, rank, "spectral", 4, stream=stream, device=dev)
        if args.peer:
            ex = S.PeerExchange(slab) if world > 1 else S.LocalPeerExchange([slab])
        else:
            ex = S.DistExchange()
        step_fn = S.step
    sampler = ClockSampler(bus_id(torch, dev))
    for _ in range(args.warmup):
        step_fn([slab], [part], ex, mass, cp, ck, DT)
    slab.check()
    slab.read_timing(reset=True)
    slab.set_timing(True)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step_fn([slab], [part], ex, mass, cp, ck, DT)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier()
    slab.set_timing(False)
    t_ms = max_over_ranks(e0.elapsed_time(e1))
    stages = slab.read_timing(reset=True)
    launches = sum(n for _, n in stages.values())
    slab.check()
    value = np_ * args.steps / (t_ms / 1e3)
    peak, peak_kind = measured_peaks()
    per_stage = {s_: {"ms_per_step": ms / args.steps, "launches": n} for s_, (ms, n) in stages.items()}
    dom = max(stages, key=lambda s_: stages[s_][0])
    # algorithmic bytes of this rank's share: the single-box byte model scaled
    # by the slab's share of the mesh and of the particles
    share = 1.0 / world
    if args.pencil and dom == "sort":
        # the pencil's staging copies: own rows out of / back into the halo
        # buffer and the kz chunks packed / unpacked, each a read and a write
        # of the rank's half-spectrum share (4 per step)
        dom_bytes = 4 * 2 * ng * ng * (ng + 2) * 4 * share
    else:
        dom_bytes = stage_bytes(dom, ng, np_, 4) * share if dom in ("deposit", "kick_drift", "bin") or \
            dom.startswith("fft_") else None
    dom_ms = stages[dom][0] / args.steps  # per step (bytes per step likewise)
    roofline = {"bound": "hbm", "kernel": dom, "peak": peak, "unit": "GB/s",
                "peak_source": f"{peak_kind} hbm_gbs (copy bandwidth)", "ms_per_launch": dom_ms,
                "launches_per_step": stages[dom][1] / args.steps,
                "achieved": dom_bytes / (dom_ms / 1e3) / 1e9 if dom_bytes else None,
                "frac": dom_bytes / (dom_ms / 1e3) / 1e9 / peak if dom_bytes else None, "traffic": None,
                "note": f"per rank; the byte model of one box times the {'pencil' if args.pencil else 'slab'}'s "
                        "share"}
    # ---- end to end: this rank's particle state from pinned host memory and
    # back every step
    host = torch.empty(part.words.shape, dtype=torch.int32, pin_memory=True)
    host.copy_(part.words)
    nbytes = part.n * 8 * 4
    # one contiguous copy per particle word and range (a strided view of
    # pinned memory would be staged through pageable memory)
    rows_dev = [part.words[w] for w in range(part.words.shape[0])]
    rows_host = [host[w] for w in range(host.shape[0])]

    D = P if args.pencil else S

    def e2e_time(mode):
        if mode == "split":
            trip = pm.hostio.SplitRoundTrip(stream, rows_dev[:4], rows_dev[4:], rows_host[:4], rows_host[4:])

            def one():
                trip.step(part.n, lambda: D.step_potential([slab], [part], ex, mass, cp),
                          finish=lambda: D.step_finish([slab], [part], ex, ck, DT), n_out=lambda: part.n)
        else:
            trip = pm.hostio.HostRoundTrip(stream, rows_dev, rows_host, serial=mode == "serial")

            def one():
                trip.step(part.n, lambda: step_fn([slab], [part], ex, mass, cp, ck, DT), lambda: part.n)

        for _ in range(max(1, args.warmup)):
            one()
        trip.finish()
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        trip.start(e0)
        for _ in range(args.steps):
            one()
        trip.finish()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1))

    te = e2e_time("split")
    te_whole = e2e_time("whole")
    te_serial = e2e_time("serial")
    e2e = {"value": np_ * args.steps / (te / 1e3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
           "d2h_bytes_per_step": nbytes, "ms_per_step": te / args.steps, "whole_step_ms_per_step": te_whole / args.steps,
           "serial_ms_per_step": te_serial / args.steps,
           "path": f"{'pencil' if args.pencil else 'slab'}.step_potential, then .step_finish (gather, kick, "
                   f"drift, migration; pm_{'pencil' if args.pencil else 'slab'}_* through the C ABI, NCCL "
                   "exchanges); every step this rank's particle words copied from pinned host memory and back on "
                   "two copy streams: cell and offsets first, velocities and ids while the potential part runs, "
                   "downloads in 16 ranges after the migration; whole_step_ms_per_step: the whole step with the "
                   "copies in ranges; serial_ms_per_step: every copy in order on the compute stream"}
    ensemble = None
    if not args.skip_ensemble:
        slab.close()
        del part, host
        torch.cuda.empty_cache()
        ensemble = ensemble_leg(pm, torch, args, world, rank, dev, stream, barrier, max_over_ranks)
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{nrow}^3 particles on {ng}^3 mesh, FP32 mesh/FFT/forces, split positions, "
                                   f"spectral Poisson, 4-point gradient, KDK dt={DT}, Zel'dovich P(k)~k^{N_S} "
                                   f"rms {RMS} cell",
                       "particles_total": np_, "mesh": ng, "l2": "inputs larger than L2",
                       "parallelism": (f"pencil{px}x{py}: pencils of {ng // px} x {ng // py} columns, one per "
                                       f"GPU; ghost rows, two y-group and two x-group all-to-all transposes, "
                                       f"two-axis potential halo, particle migration" if args.pencil else
                                       f"slab{world}: x-slabs of {ng // world} planes, one per GPU; NCCL ghost "
                                       f"fold, two " + ("transposes by the FFT kernels' stores into the other "
                                                        "GPUs' memory" if args.peer else "all-to-all transposes")
                                       + ", potential halo, particle migration")},
            "stages": per_stage, "ensemble": ensemble, "e2e": e2e, "roofline": roofline, "cpu_baseline": None,
            "clocks": clocks, "gpu_launches": launches}
    print(json.dumps(line), flush=True)
    return 0


# -------------------------------------------------------------- GPU side
def ours(args):
    import torch
    import torch.distributed as dist
    from loader import load_package

    pm = load_package()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        return reduce_max(v, world, dev)

    ng, nrow = args.ng, args.nrow
    np_ = nrow ** 3
    mass = ng ** 3 / np_
    cp, ck = pm.unit_box_coefficients(DT)
    stream = torch.cuda.current_stream(dev)
    if world > 1 or args.slab or args.pencil or args.peer:
        return ours_slab(args, pm, torch, dist, world, rank, dev, stream, barrier, max_over_ranks)

    pos, vel = pm.zeldovich_ic(ng, nrow, N_S, RMS, rank_seed(rank), device=dev)
    p32 = pm.Plan(ng, "fp32", "spectral", 4, stream=stream, device=dev)
    if args.gather != "cached":
        p32.set_gather(args.gather)
    cell, off = p32.split(*pos)
    v32 = [a.float() for a in vel]
    torch.cuda.synchronize()

    # nvidia-smi takes a moment to start: launch the sampler before the
    # warm-up so that it samples the whole timed region
    sampler = ClockSampler(bus_id(torch, dev))
    for _ in range(args.warmup):
        p32.step_split(cell, off, v32, mass, cp, ck, DT)
    p32.check()
    p32.read_timing(reset=True)
    p32.set_timing(True)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        p32.step_split(cell, off, v32, mass, cp, ck, DT)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier()
    p32.set_timing(False)
    t_ms = max_over_ranks(e0.elapsed_time(e1))
    stages = p32.read_timing(reset=True)
    p32.check()
    value = throughput(world, np_, args.steps, t_ms)
    launches = sum(n for _, n in stages.values())

    # every stage runs once per step (binning is five kernel launches, every
    # other stage one), so bytes and times are per step, launches counted apart
    peak, peak_kind = measured_peaks()
    dom = max(stages, key=lambda s: stages[s][0])
    dom_ms = stages[dom][0] / args.steps
    dom_bytes = stage_bytes(dom, ng, np_, 4)
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    traffic = ncu_traffic(dom, ng)
    step_bytes = sum(stage_bytes(s, ng, np_, 4) for s in stages)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs (copy bandwidth)",
                "traffic": traffic, "algorithmic_bytes_per_launch": dom_bytes, "ms_per_launch": dom_ms,
                "step": {"algorithmic_bytes": step_bytes, "achieved": step_bytes / (t_ms / args.steps / 1e3) / 1e9,
                         "frac": step_bytes / (t_ms / args.steps / 1e3) / 1e9 / peak}}
    per_stage = {s: {"ms_per_step": ms / args.steps, "launches": n,
                     "gbs": stage_bytes(s, ng, np_, 4) * args.steps / (ms / 1e3) / 1e9 if ms > 0 else None}
                 for s, (ms, n) in stages.items()}

    # ---- FP64 plain path on the same initial state + force error
    fp64 = None
    force_err = None
    fp64_size_ok = True  # the plain FP64 path takes every mesh size the FP32 one does
    if not args.skip_fp64 and fp64_size_ok:
        p64 = pm.Plan(ng, "fp64", "spectral", 4, stream=stream, device=dev)
        x, y, z = (a.clone() for a in pos)
        pv = [a.clone() for a in vel]
        # forces at the initial state through the timed kernels: the fused
        # FP32 step (pm_step_f32) with zero velocities, c_kick = 1 and dt = 0
        # returns the forces in v; the FP64 step does the same into p
        zero = [torch.zeros_like(x) for _ in range(3)]
        p64.step(x, y, z, *zero, mass, cp, 1.0, 0.0)
        c0, o0 = p32.split(*pos)
        f32 = [torch.zeros_like(o0[0]) for _ in range(3)]
        p32.step_split(c0, o0, f32, mass, cp, 1.0, 0.0)
        num = sum(float(((a.double() - b) ** 2).sum()) for a, b in zip(f32, zero))
        den = sum(float((b ** 2).sum()) for b in zero)
        force_err = math.sqrt(num / den)
        del zero, c0, o0, f32
        for _ in range(args.warmup):
            p64.step(x, y, z, *pv, mass, cp, ck, DT)
        p64.read_timing(reset=True)
        p64.set_timing(True)
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            p64.step(x, y, z, *pv, mass, cp, ck, DT)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        t64 = max_over_ranks(e0.elapsed_time(e1))
        st64 = p64.read_timing(reset=True)
        b64 = sum(stage_bytes(s, ng, np_, 8) for s in st64)
        fp64 = {"value": throughput(world, np_, args.steps, t64), "unit": UNIT, "ms_per_step": t64 / args.steps,
                "roofline": {"bound": "hbm", "algorithmic_bytes_per_step": b64,
                             "achieved": b64 / (t64 / args.steps / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": b64 / (t64 / args.steps / 1e3) / 1e9 / peak},
                "dtype": "f64", "path": "plain FP64: separate deposit, 3+3 FFT passes, Green, gradient to 3 force "
                                        "meshes, interpolate + kick, drift",
                "stages": {s: {"ms_per_step": ms / args.steps, "launches": n,
                               "gbs": stage_bytes(s, ng, np_, 8) * args.steps / (ms / 1e3) / 1e9 if ms > 0 else None}
                           for s, (ms, n) in st64.items()}}
        p64.close()
        del p64, x, y, z, pv
        torch.cuda.empty_cache()

    # ---- accuracy of the FP32 split path against the FP64 path over the
    # configuration's own run: 50 leapfrog KDK steps at dt = 0.005 from the
    # same initial state (half kicks merged; 51 force evaluations)
    accuracy = None
    if not args.skip_fp64 and fp64_size_ok and not args.skip_accuracy:
        nsteps = ACC_STEPS
        sched = [(0.5 * DT if s in (0, nsteps) else DT, DT if s < nsteps else 0.0) for s in range(nsteps + 1)]
        c32, o32 = p32.split(*pos)
        w32 = [a.float() for a in vel]
        x64 = [a.clone() for a in pos]
        w64 = [a.clone() for a in vel]
        p64 = pm.Plan(ng, "fp64", "spectral", 4, stream=stream, device=dev)
        m0_32 = p32.conserved(None, w32, mass)["momentum"]
        m0_64 = p64.conserved(None, w64, mass)["momentum"]
        scale = mass * float(sum(a.abs().sum() for a in vel))
        for ckk, dd in sched:
            p32.step_split(c32, o32, w32, mass, cp, ckk, dd)
            p64.step(*x64, *w64, mass, cp, ckk, dd)
        p32.check()
        p64.check()
        xj = p32.join(c32, o32)
        d2, dmax = 0.0, 0.0
        for a, b in zip(xj, x64):
            d = torch.remainder(a - b + 0.5 * ng, float(ng)) - 0.5 * ng
            d2 += float((d * d).sum())
            dmax = max(dmax, float(d.abs().max()))
        vnum = sum(float(((a.double() - b) ** 2).sum()) for a, b in zip(w32, w64))
        vden = sum(float((b ** 2).sum()) for b in w64)
        dens32 = p32.deposit_split(c32, o32, mass, p32.workspace_mesh())
        c_32 = p32.conserved(dens32, w32, mass)
        dens32 = dens32[:, :, :ng].double()
        dens64 = p64.deposit(*x64, mass)
        c_64 = p64.conserved(dens64, w64, mass)
        dens64 = dens64[:, :, :ng]
        dnum = float(((dens32 - dens64) ** 2).sum())
        dden = float(((dens64 + 1.0) ** 2).sum())
        accuracy = {"steps": nsteps, "dt": DT, "schedule": "leapfrog KDK, half kicks merged",
                    "force_rel_l2_initial": force_err,
                    "position_err_rms_cells": math.sqrt(d2 / (3 * np_)), "position_err_max_cells": dmax,
                    "velocity_rel_l2": math.sqrt(vnum / vden),
                    "density_rel_l2": math.sqrt(dnum / dden),
                    "mass_rel_err": {"fp32": c_32["mass"] / (mass * np_) - 1.0,
                                     "fp64": c_64["mass"] / (mass * np_) - 1.0},
                    "momentum_drift_rel": {
                        "fp32": max(abs(a - b) for a, b in zip(c_32["momentum"], m0_32)) / scale,
                        "fp64": max(abs(a - b) for a, b in zip(c_64["momentum"], m0_64)) / scale},
                    "note": "FP32 vs FP64 from the same seed; mass and momentum summed in FP64 on the device; "
                            "density error relative to the FP64 density 1 + delta"}
        p64.close()
        del p64, x64, w64, c32, o32, w32, xj, dens32, dens64
        torch.cuda.empty_cache()

    # ---- adjoint step vs forward step, differentiable-PM configuration
    # (128^3 on 128^3; the FP32 split path is the configuration's own, FP64
    # its check path)
    adjoint = None
    if not args.skip_adjoint:
        na = 128
        pa, va = pm.zeldovich_ic(na, na, -2.0, 0.5, 7 + rank, device=dev)

        def timed(fn, reps=20):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps

        def leg(t_f, t_a, prec):
            return {"config": f"128^3 particles on 128^3 mesh, {prec}, spectral Poisson, 4-point gradient",
                    "forward_step_ms": t_f, "adjoint_step_ms": t_a, "adjoint_over_forward": t_a / t_f,
                    "with_recompute_over_forward": (t_a + t_f) / t_f}

        p32a = pm.Plan(na, "fp32", "spectral", 4, stream=stream, device=dev)
        acell, aoff = p32a.split(*pa)
        av32 = [a.float().contiguous() for a in va]
        cs, os_, vs32 = acell.clone(), [a.clone() for a in aoff], [a.clone() for a in av32]
        xb32 = [torch.randn_like(aoff[0]) for _ in range(3)]
        vb32 = [torch.randn_like(aoff[0]) for _ in range(3)]
        t_f32 = timed(lambda: p32a.step_split(cs, os_, vs32, 1.0, cp, 0.01, 0.01))
        t_a32 = timed(lambda: p32a.step_adjoint_split(acell, aoff, 1.0, cp, 0.01, 0.01, xb32, vb32))
        adjoint = leg(t_f32, t_a32, "FP32 split positions")
        adjoint["note"] = ("adjoint step = force recomputation at the step's start + transposed pairs; "
                           "checkpointed backprop also re-runs each forward step once")
        p32a.close()
        del p32a, acell, aoff, av32, cs, os_, vs32, xb32, vb32
        if not args.skip_fp64:
            pla = pm.Plan(na, "fp64", "spectral", 4, stream=stream, device=dev)
            xb = [torch.randn_like(pa[0]) for _ in range(3)]
            vb = [torch.randn_like(pa[0]) for _ in range(3)]
            xs = [a.clone() for a in pa]
            vs = [a.clone() for a in va]
            t_f = timed(lambda: pla.step(*xs, *vs, 1.0, cp, 0.01, 0.01))
            t_a = timed(lambda: pla.step_adjoint(*pa, 1.0, cp, 0.01, 0.01, xb, vb))
            adjoint["fp64"] = leg(t_f, t_a, "FP64")
            pla.close()
            del pla, xb, vb, xs, vs
        del pa, va

    # ---- the FP64 configuration checked against the reference: 256^3
    # particles on a 256^3 mesh, P(k) ~ k^-2, rms 0.5 cell, 20 KDK steps at
    # dt = 0.01 (parity with the reference is in the tests; this times it)
    c2 = None
    if not args.skip_fp64:
        n2 = 256
        pos2, vel2 = pm.zeldovich_ic(n2, n2, -2.0, 0.5, 21 + rank, device=dev)
        p2 = pm.Plan(n2, "fp64", "spectral", 4, stream=stream, device=dev)
        s2, d2 = 20, 0.01
        sched2 = [(0.5 * d2 if s in (0, s2) else d2, d2 if s < s2 else 0.0) for s in range(s2 + 1)]
        p2.step(*pos2, *vel2, 1.0, cp, 0.0, 0.0)  # warm-up (no kick, no drift)
        torch.cuda.synchronize()
        e0.record(stream)
        for ckk, dd in sched2:
            p2.step(*pos2, *vel2, 1.0, cp, ckk, dd)
        e1.record(stream)
        torch.cuda.synchronize()
        p2.check()
        t2 = e0.elapsed_time(e1)
        c2 = {"config": "256^3 particles on 256^3 mesh, FP64, P(k)~k^-2, rms 0.5 cell, 20 KDK steps dt=0.01 "
                        "(21 force evaluations)",
              "value": n2 ** 3 * len(sched2) / (t2 / 1e3), "unit": UNIT, "ms_per_step": t2 / len(sched2)}
        p2.close()
        del p2, pos2, vel2
        torch.cuda.empty_cache()

    # ---- batched ensemble: 256 boxes of mixed mesh sizes, 20 KDK steps per graph
    ensemble = None
    if not args.skip_ensemble:
        ensemble = ensemble_leg(pm, torch, args, world, rank, dev, stream, barrier, max_over_ranks)

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.skip_e2e:
        host = [torch.empty(np_, dtype=t.dtype, pin_memory=True) for t in [cell, *off, *v32]]
        for h, d in zip(host, [cell, *off, *v32]):
            h.copy_(d)
        dbuf = [cell, *off, *v32]
        nbytes = sum(h.numel() * h.element_size() for h in host)

        def e2e_time(mode):
            if mode == "split":
                trip = pm.hostio.SplitRoundTrip(stream, dbuf[:4], dbuf[4:], host[:4], host[4:])

                def one():
                    trip.step(np_, lambda: p32.potential_split(cell, off, mass, cp),
                              lambda lo, hi: p32.kick_drift_split(p32.workspace_mesh(), cell[lo:hi],
                                                                  [a[lo:hi] for a in off], [a[lo:hi] for a in v32],
                                                                  ck, DT))
            else:
                trip = pm.hostio.HostRoundTrip(stream, dbuf, host, serial=mode == "serial")

                def one():
                    trip.step(np_, lambda: p32.step_split(cell, off, v32, mass, cp, ck, DT))

            for _ in range(max(1, args.warmup)):
                one()
            trip.finish()
            barrier()
            torch.cuda.synchronize()
            e0.record(stream)
            trip.start(e0)
            for _ in range(args.steps):
                one()
            trip.finish()
            e1.record(stream)
            torch.cuda.synchronize()
            barrier()
            return max_over_ranks(e0.elapsed_time(e1))

        te = e2e_time("split")
        te_whole = e2e_time("whole")
        te_serial = e2e_time("serial")
        e2e = {"value": throughput(world, np_, args.steps, te), "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "ms_per_step": te / args.steps,
               "whole_step_ms_per_step": te_whole / args.steps, "serial_ms_per_step": te_serial / args.steps,
               "path": "pm_potential_f32 then pm_kick_drift_f32 over 16 particle ranges (the two halves of "
                       "pm_step_f32, same result) through the C ABI; every step all seven words of every particle "
                       "copied from pinned host memory and the new state back on two copy streams: positions "
                       "first, velocities after them (uploaded while the potential is computed), each range "
                       "downloaded when its gather is done and uploaded again for the next step after its "
                       "download; whole_step_ms_per_step: pm_step_f32 with the same copies in 16 ranges; "
                       "serial_ms_per_step: every copy one after another on the compute stream"}
        del host

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        r = cpu_reference_steps(3, 1, budget_s=30.0)
        ng_s, nrow_s = CPU_SAMPLE
        cpu = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "omp_threads": r["omp_threads"],
               "kind": r["kind"],
               "sample": f"{nrow_s}^3 particles on a {ng_s}^3 periodic mesh (1/64 of the workload: one rank's "
                         f"share of a 64-rank run), {r['steps']} steps of {r['seconds']:.3f} s; reference kernels "
                         f"(oracle/_ref) on {r['omp_threads']} OpenMP threads, scipy.fft on all cores standing in "
                         f"for FFTW"}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    # Key order: the bulky detail first, the metric's own figures last (a
    # reader of the line's tail sees the FP64 half of the metric, the speed-up,
    # the force error and the 50-step accuracy).
    fp64_head = None
    if fp64 and "value" in fp64:
        fp64_head = {"value": fp64["value"], "ms_per_step": fp64["ms_per_step"],
                     "roofline_frac": fp64["roofline"]["frac"], "path": "plain FP64 (pm_step_f64)"}
    elif fp64:
        fp64_head = fp64
    acc_head = None
    if accuracy:
        acc_head = {k: accuracy[k] for k in ("steps", "dt", "position_err_rms_cells", "position_err_max_cells",
                                              "velocity_rel_l2", "density_rel_l2")}
        acc_head["mass_rel_err_fp32"] = accuracy["mass_rel_err"]["fp32"]
        acc_head["momentum_drift_rel_fp32"] = accuracy["momentum_drift_rel"]["fp32"]
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{nrow}^3 particles on {ng}^3 mesh, FP32 mesh/FFT/forces, split positions, "
                                   f"spectral Poisson, 4-point gradient, KDK dt={DT}, Zel'dovich P(k)~k^{N_S} "
                                   f"rms {RMS} cell",
                       "particles_per_gpu": np_, "mesh": ng, "l2": "inputs larger than L2 (mesh 4.3 GB)",
                       "particle_order": "Lagrangian (lattice) order as generated; the deposit re-bins every "
                                         "step",
                       "gather": args.gather,
                       "parallelism": f"{world} independent boxes, one per GPU"},
            "stages": per_stage, "fp64_detail": fp64, "accuracy_detail": accuracy, "fp64_256": c2,
            "adjoint": adjoint, "ensemble": ensemble,
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches,
            "fp64": fp64_head,
            "speedup_fp32_vs_fp64": (value / fp64["value"]) if fp64 and "value" in fp64 else None,
            "force_err": force_err,
            "force_err_path": "pm_step_f32 (the timed fused kernels) vs pm_step_f64, v=0, c_kick=1, dt=0",
            "accuracy": acc_head}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
