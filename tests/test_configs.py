"""Parity at the configurations the path is specified on, through the C ABI.

  C1  64^3 particles on a 64^3 mesh, Zel'dovich P(k) ~ k^-2, rms 0.3 cell,
      10 leapfrog KDK steps at dt = 0.01, spectral Poisson, 4-point gradient:
      the FP64 GPU path against the CPU oracle.
  C2  256^3 particles on a 256^3 mesh, P(k) ~ k^-2, rms 0.5 cell, 20 KDK
      steps at dt = 0.01: the FP64 GPU path against the CPU oracle.
  C3  512^3 (and 128^3) particles on a 1024^3 mesh, P(k) ~ k^-1.5, rms 1 cell:
      the forces of the fused FP32 step (pm_step_f32 with zero velocities,
      c_kick = 1, dt = 0, so v comes back as the force) against the FP64 step.
  FFT 1024^3 R2C of both precisions against cuFFT (torch.fft.rfftn in FP64),
      cuFFT only as the independent cross-check.

Tolerances (relative L2, written in each assertion):
  FP64 GPU vs oracle: 1e-12 on density, potential, forces, velocities and
  final positions (positions also relative to the displacement itself);
  FP32 fused step vs FP64: forces 1e-4 (the mixed-precision target);
  FFT: FP64 1e-13, FP32 2e-6.
The oracle (oracle/pm_oracle.c + numpy.fft, pinned against the compiled
reference in tests/test_oracle.py) runs on the host CPU beside the GPU.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def H(t):
    return t.detach().cpu().numpy()


def periodic_diff(a, b, ng):
    d = np.asarray(a, np.float64) - np.asarray(b, np.float64)
    return d - ng * np.round(d / ng)


def lattice(ng, nrow):
    q = (np.arange(nrow) + 0.5) * (ng / nrow)
    qx, qy, qz = np.meshgrid(q, q, q, indexing="ij")
    return [qx.ravel(), qy.ravel(), qz.ravel()]


def kdk_vs_oracle(pmpkg, O, ng, nrow, n_s, rms, seed, steps, dt):
    """Runs the same KDK schedule on the GPU FP64 plan and in the oracle from
    one initial state; returns the errors of the final state."""
    cp, mass, kind, order = 4 * np.pi, ng ** 3 / nrow ** 3, 1, 4
    gpos, gvel = pmpkg.zeldovich_ic(ng, nrow, n_s, rms, seed=seed, device=DEV)
    pos0 = [H(a) for a in gpos]
    vel0 = [H(a) for a in gvel]
    out = {}

    # forces at the initial state (identical inputs on both sides)
    plan = pmpkg.Plan(ng, "fp64", "spectral", order)
    zero = [torch.zeros_like(gpos[0]) for _ in range(3)]
    plan.step(*(a.clone() for a in gpos), *zero, mass, cp, 1.0, 0.0)
    f0 = [np.zeros(nrow ** 3) for _ in range(3)]
    d0, phi0, _ = O.force_step(ng, *(a.copy() for a in pos0), *f0, mass, cp, 1.0, kind, order)
    out["force0"] = rel(np.stack([H(a) for a in zero]), np.stack(f0))
    out["potential0"] = rel(H(plan.workspace_mesh())[:, :, :ng], phi0[:, :, :ng])
    out["density0"] = rel(H(plan.deposit(*gpos, mass))[:, :, :ng], d0[:, :, :ng])

    # the KDK run: steps + 1 force evaluations, inner half kicks merged
    x, v = [a.copy() for a in pos0], [a.copy() for a in vel0]
    tx, tv = [a.clone() for a in gpos], [a.clone() for a in gvel]
    for s in range(steps + 1):
        ck = 0.5 * dt if s in (0, steps) else dt
        dd = dt if s < steps else 0.0
        plan.step(*tx, *tv, mass, cp, ck, dd)
        delta, phi, _ = O.force_step(ng, *x, *v, mass, cp, ck, kind, order)
        if s < steps:
            O.drift(ng, *x, *v, dt)
    plan.check()
    # the last force evaluation ran at the final positions (no drift after it)
    out["potential"] = rel(H(plan.workspace_mesh())[:, :, :ng], phi[:, :, :ng])
    out["density"] = rel(H(plan.deposit(*tx, mass))[:, :, :ng], delta[:, :, :ng])
    out["velocity"] = rel(np.stack([H(a) for a in tv]), np.stack(v))
    dx = np.stack([periodic_diff(H(a), b, ng) for a, b in zip(tx, x)])
    out["position"] = float(np.linalg.norm(dx) / np.linalg.norm(np.stack(x)))
    disp = np.stack([periodic_diff(b, q, ng) for b, q in zip(x, lattice(ng, nrow))])
    out["position_vs_displacement"] = float(np.linalg.norm(dx) / np.linalg.norm(disp))
    out["position_max_cells"] = float(np.abs(dx).max())
    return out


def test_c1_plain_pm_64_matches_oracle(pmpkg, O):
    """C1: 64^3 on 64^3, P(k) ~ k^-2, rms 0.3 cell, 10 KDK steps at dt = 0.01;
    the GPU initial conditions equal the oracle's, and the FP64 GPU run
    matches the oracle's to 1e-12."""
    gpos, gvel = pmpkg.zeldovich_ic(64, 64, -2.0, 0.3, seed=101, device=DEV)
    opos, ovel = O.zeldovich_ic(64, 64, -2.0, 0.3, seed=101)
    assert rel(np.stack([H(a) for a in gvel]), np.stack(ovel)) < 1e-12
    assert max(np.abs(periodic_diff(H(a), b, 64)).max() for a, b in zip(gpos, opos)) < 1e-11
    e = kdk_vs_oracle(pmpkg, O, 64, 64, -2.0, 0.3, 101, 10, 0.01)
    print("C1", e)
    for k in ("force0", "potential0", "density0", "potential", "density", "velocity", "position",
              "position_vs_displacement"):
        assert e[k] < 1e-12, (k, e[k])


def test_c2_plain_pm_256_matches_oracle(pmpkg, O):
    """C2: 256^3 on 256^3, P(k) ~ k^-2, rms 0.5 cell, 20 KDK steps at
    dt = 0.01: density, potential, forces, velocities and final positions of
    the FP64 GPU run within 1e-12 (relative L2) of the oracle's."""
    e = kdk_vs_oracle(pmpkg, O, 256, 256, -2.0, 0.5, 202, 20, 0.01)
    print("C2", e)
    for k in ("force0", "potential0", "density0", "potential", "density", "velocity", "position",
              "position_vs_displacement"):
        assert e[k] < 1e-12, (k, e[k])
    torch.cuda.empty_cache()


@pytest.mark.parametrize("nrow", [128, 512])
def test_c3_fused_fp32_step_forces_within_1e4_of_fp64(pmpkg, nrow):
    """C3 at full size through the timed kernels: pm_step_f32 (binning, the
    deposit fused with the z R2C, y / x + Green / y passes through the
    transposed spectrum, z C2R, fused gradient + gather + kick) with zero
    velocities, c_kick = 1 and dt = 0 returns the FP32 forces in v; the FP64
    step does the same into p.  Relative L2 <= 1e-4, and the FP32 potential
    within 1e-4 of the FP64 one."""
    ng = 1024
    mass, cp = ng ** 3 / nrow ** 3, 4 * np.pi
    pos, vel = pmpkg.zeldovich_ic(ng, nrow, -1.5, 1.0, seed=303, device=DEV)
    del vel
    p32 = pmpkg.Plan(ng, "fp32", "spectral", 4)
    cell, off = p32.split(*pos)
    v32 = [torch.zeros_like(off[0]) for _ in range(3)]
    p32.step_split(cell, off, v32, mass, cp, 1.0, 0.0)
    p32.check()
    phi32 = p32.workspace_mesh()[:, :, :ng].clone()
    p32.close()
    del p32, cell, off
    torch.cuda.empty_cache()
    p64 = pmpkg.Plan(ng, "fp64", "spectral", 4)
    f64 = [torch.zeros_like(pos[0]) for _ in range(3)]
    p64.step(*pos, *f64, mass, cp, 1.0, 0.0)
    p64.check()
    phi64 = p64.workspace_mesh()[:, :, :ng]
    perr = float((phi32.double() - phi64).norm() / phi64.norm())
    num = sum(float(((a.double() - b) ** 2).sum()) for a, b in zip(v32, f64))
    den = sum(float((b ** 2).sum()) for b in f64)
    ferr = (num / den) ** 0.5
    print(f"C3 nrow={nrow}: force rel L2 {ferr:.3e}, potential rel L2 {perr:.3e}")
    assert ferr <= 1e-4, ferr
    assert perr <= 1e-4, perr
    p64.close()
    del p64, phi32, phi64, f64, v32, pos
    torch.cuda.empty_cache()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_fft_1024_against_cufft(pmpkg, prec):
    """The hand-written 1024^3 R2C of either precision against cuFFT
    (torch.fft.rfftn of the same input in FP64): FP64 within 1e-13, FP32
    within 2e-6 (relative L2 over the half spectrum)."""
    ng = 1024
    g = torch.Generator(device=DEV).manual_seed(1024 + (prec == "fp32"))
    plan = pmpkg.Plan(ng, prec)
    d = plan.new_mesh()
    d[:, :, :ng] = torch.randn((ng, ng, ng), generator=g, device=DEV, dtype=d.dtype)
    ref = torch.fft.rfftn(d[:, :, :ng].double())
    plan.fft_r2c(d)
    ours = torch.view_as_complex(d.view(ng, ng, ng // 2 + 1, 2))
    err = float((ours.to(torch.complex128) - ref).abs().norm() / ref.abs().norm())
    del ours, ref, d
    torch.cuda.empty_cache()
    print(f"1024^3 {prec} R2C vs cuFFT: rel L2 {err:.3e}")
    assert err < (1e-13 if prec == "fp64" else 2e-6), err
