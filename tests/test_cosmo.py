"""Cosmological time stepping (leapfrog KDK in the scale factor) and the
snapshot format.  The schedule of the Python and C++ mirrors agree; the FP64
GPU run matches the oracle's restatement; the FP32 split path tracks the FP64
path; snapshots round-trip between the Python reader / writer and the C++
writer of pm_main."""
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden

DRV = os.path.join(ROOT, "particle-mesh_b200", "driver")


def test_schedule_formulas(pmpkg):
    pm = pmpkg
    a0, da, n = 0.9, 0.01, 4
    sch = pm.cosmo_schedule(a0, da, n)
    assert len(sch) == n + 1
    for s, (a, cp, ck, dt) in enumerate(sch):
        assert a == pytest.approx(a0 + s * da, rel=1e-15)
        assert cp == pytest.approx(1.5 / a, rel=1e-15)
        w = 0.5 if s in (0, n) else 1.0
        assert ck == pytest.approx(w * pm.function_a(a) * da, rel=1e-15)
        if s < n:
            ah = a0 + (s + 0.5) * da
            assert dt == pytest.approx(pm.function_a(ah) * da / ah ** 2, rel=1e-15)
        else:
            assert dt == 0.0


def test_schedule_matches_cpp_mirror(pmpkg, tmp_path):
    pm = pmpkg
    src = tmp_path / "cs.cpp"
    src.write_text('#include <cstdio>\n#include "pm_b200.hpp"\n'
                   'int main(){ for (auto& c : pm::cosmo_schedule(0.9, 0.01, 6))'
                   ' { double v[4] = {c.a, c.c_poisson, c.c_kick, c.dt}; fwrite(v, 8, 4, stdout); } }\n')
    exe = tmp_path / "cs"
    subprocess.run(["g++", "-std=c++17", "-O0", "-I", os.path.join(ROOT, "include"), "-I", DRV, str(src), "-o",
                    str(exe)], check=True)
    out = np.frombuffer(subprocess.run([str(exe)], capture_output=True, check=True).stdout, np.float64)
    ref = np.array(pm.cosmo_schedule(0.9, 0.01, 6)).ravel()
    assert np.allclose(out, ref, rtol=1e-15, atol=0)


def test_snapshot_round_trip_and_cpp_writer(pmpkg, tmp_path):
    import torch
    pm = pmpkg
    rng = np.random.default_rng(4)
    arrs = [torch.tensor(rng.uniform(0, 16, 300)) for _ in range(6)]
    f = tmp_path / "s.bin"
    pm.write_snapshot(str(f), 16, 0.95, 1.5, arrs[:3], [a.float() for a in arrs[3:]])
    d = pm.read_snapshot(str(f))
    assert (d["ng"], d["np"], d["a"], d["mass"]) == (16, 300, 0.95, 1.5)
    assert all(torch.equal(a, b) for a, b in zip(d["pos"], arrs[:3]))
    assert all(torch.equal(a.float().double(), b) for a, b in zip(arrs[3:], d["vel"]))
    assert os.path.getsize(f) == 72 + 6 * 8 * 300
    # the C++ writer produces the same bytes for the same data
    src = tmp_path / "ws.cpp"
    src.write_text('#include <vector>\n#include "pm_b200.hpp"\n'
                   'int main(int, char** argv){ size_t n = 5; std::vector<double> v[6];\n'
                   ' for (int c = 0; c < 6; ++c) for (size_t i = 0; i < n; ++i) v[c].push_back(c * 10.0 + i);\n'
                   ' const double* h[6]; for (int c = 0; c < 6; ++c) h[c] = v[c].data();\n'
                   ' pm::write_snapshot(argv[1], 32, 0.91, 8.0, h, n); }\n')
    exe = tmp_path / "ws"
    subprocess.run(["g++", "-std=c++17", "-O0", "-I", os.path.join(ROOT, "include"), "-I", DRV, str(src), "-o",
                    str(exe)], check=True)
    g = tmp_path / "c.bin"
    subprocess.run([str(exe), str(g)], check=True)
    d = pm.read_snapshot(str(g))
    assert (d["ng"], d["np"], d["a"], d["mass"]) == (32, 5, 0.91, 8.0)
    for c in range(6):
        t = (d["pos"] + d["vel"])[c]
        assert t.tolist() == [c * 10.0 + i for i in range(5)]
    p = tmp_path / "p.bin"
    pm.write_snapshot(str(p), 32, 0.91, 8.0, [torch.tensor([c * 10.0 + i for i in range(5)]) for c in range(3)],
                      [torch.tensor([c * 10.0 + i for i in range(5)]) for c in range(3, 6)])
    assert p.read_bytes() == g.read_bytes()


def test_snapshot_reader_rejects_bad_files(pmpkg, tmp_path):
    pm = pmpkg
    f = tmp_path / "bad.bin"
    f.write_bytes(b"NOTASNAP" + bytes(64))
    with pytest.raises(pm.PMError):
        pm.read_snapshot(str(f))
    f.write_bytes(struct.pack("<8sIIqqddddd", b"PMSNAP1\0", 1, 0, 8, 10, 1.0, 1.0, 0.3, 0.7, 1.0) + bytes(16))
    with pytest.raises(pm.PMError):
        pm.read_snapshot(str(f))


# ------------------------------------------------------------------ GPU
def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
def test_cosmo_run_fp64_matches_oracle_and_fp32_tracks(pmpkg, O):
    torch = _cuda()
    ng, nrow, n, da = 32, 16, 20, 0.01
    pos, vel = O.zeldovich_ic(ng, nrow, -2.0, 0.5, seed=31)
    mass = ng ** 3 / nrow ** 3
    x, y, z = (a.copy() for a in pos)
    px, py, pz = (a.copy() for a in vel)
    O.cosmo_kdk(ng, x, y, z, px, py, pz, mass, 0.9, da, n, 0, 2)
    T = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")  # noqa: E731
    plan = pmpkg.Plan(ng, "fp64", "discrete", 2)
    gp, gv = [T(a) for a in pos], [T(a) for a in vel]
    a_end = pmpkg.cosmo_run(plan, gp, gv, mass, 0.9, da, n)
    assert a_end == pytest.approx(0.9 + n * da)
    got = np.stack([a.cpu().numpy() for a in gp])
    d = got - np.stack([x, y, z])
    d -= ng * np.round(d / ng)
    assert np.abs(d).max() < 1e-10
    mom = np.stack([a.cpu().numpy() for a in gv])
    ref = np.stack([px, py, pz])
    assert np.linalg.norm(mom - ref) / np.linalg.norm(ref) < 1e-11
    # the FP32 split path over the same schedule
    p32 = pmpkg.Plan(ng, "fp32", "discrete", 2)
    cell, off = p32.split(*(T(a) for a in pos))
    v32 = [T(a, torch.float32) for a in vel]
    pmpkg.cosmo_run(p32, (cell, off), v32, mass, 0.9, da, n)
    j = np.stack([a.cpu().numpy() for a in p32.join(cell, off)])
    d = j - got
    d -= ng * np.round(d / ng)
    assert np.abs(d).max() < 1e-4


@pytest.mark.gpu
def test_driver_cosmo_snapshot(pmpkg, tmp_path):
    torch = _cuda()
    exe = os.path.join(ROOT, "particle-mesh_b200", "pm_main")
    if not os.path.exists(exe):
        pytest.skip("pm_main not built")
    snap = tmp_path / "snap.bin"
    r = subprocess.run([exe, "16", "16", "--steps", "0", "--warmup", "0", "--cosmo", "5", "--snapshot", str(snap)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    d = pmpkg.read_snapshot(str(snap))
    assert (d["ng"], d["np"]) == (16, 16 ** 3)
    assert d["a"] == pytest.approx(0.9 + 5 * 0.001)
    # the same run through the Python mirror from pm_main's initial state
    g = load_golden("ref_step_ng16_np16.npz")
    pos = [torch.tensor(g["pos"][i], device="cuda") for i in range(3)]
    mom = [torch.zeros(16 ** 3, dtype=torch.float64, device="cuda") for _ in range(3)]
    plan = pmpkg.Plan(16, "fp64", "discrete", 2)
    pmpkg.cosmo_run(plan, pos, mom, 1.0, nsteps=5)
    # equal to rounding (the FP64 deposit's atomic adds have no fixed order)
    for a, b in zip(pos + mom, d["pos"] + d["vel"]):
        assert float((a.cpu() - b).norm() / b.norm()) < 1e-12
