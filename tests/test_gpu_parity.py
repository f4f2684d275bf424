"""GPU parity of every stage of the particle-mesh step against the CPU oracle.

Tolerances (relative L2 unless stated):
  FP64 path vs oracle / golden fixtures:  1e-12 (density 1e-13)
  FP32 split path vs the FP64 oracle:     forces 1e-4 (the target), potential 1e-4
All calls go through the C ABI (libpm_b200.so) via the package's ctypes layer.
"""
import numpy as np
import pytest

from conftest import golden_cases, load_golden

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    a = a.astype(np.complex128 if np.iscomplexobj(a) else np.float64)
    b = b.astype(np.complex128 if np.iscomplexobj(b) else np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def T(a, dtype=torch.float64):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def H(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def uniform(ng, n, seed):
    rng = np.random.default_rng(seed)
    return [rng.uniform(0, ng, n) for _ in range(3)]


# ------------------------------------------------------------------- FFT

@pytest.mark.parametrize("ng", [8, 16, 32, 64, 128])
def test_fft_r2c_c2r_f64(pmpkg, O, ng):
    rng = np.random.default_rng(ng)
    m = O.padded(ng)
    m[:, :, :ng] = rng.standard_normal((ng, ng, ng))
    plan = pmpkg.Plan(ng, "fp64")
    d = T(m)
    plan.fft_r2c(d)
    spec = H(d).view(np.complex128)
    ref = np.fft.rfftn(m[:, :, :ng])
    assert rel(spec, ref) < 1e-13
    if ng <= 32:
        mm = m.copy()
        O.rfft3d_forward(mm)
        assert rel(spec, O.spectrum_view(mm)) < 1e-13
    plan.fft_c2r(d)
    assert rel(H(d)[:, :, :ng], ng ** 3 * m[:, :, :ng]) < 1e-13
    assert np.all(H(d)[:, :, ng:] == 0)


@pytest.mark.parametrize("ng", [256, 512])
def test_fft_round_trip_large_f64(pmpkg, ng):
    g = torch.Generator(device=DEV).manual_seed(ng)
    plan = pmpkg.Plan(ng, "fp64")
    d = plan.new_mesh()
    d[:, :, :ng] = torch.randn((ng, ng, ng), generator=g, device=DEV, dtype=torch.float64)
    x = d[:, :, :ng].clone()
    plan.fft_r2c(d)
    # Parseval for the half spectrum: sum|x|^2 N^3 = |X0|^2 + 2 sum_mid |X|^2 + |XN|^2
    s = torch.view_as_complex(d.view(ng, ng, ng // 2 + 1, 2))
    e = (s[:, :, 0].abs() ** 2).sum() + (s[:, :, -1].abs() ** 2).sum() + 2 * (s[:, :, 1:-1].abs() ** 2).sum()
    assert float(e / ((x * x).sum() * ng ** 3)) == pytest.approx(1.0, abs=1e-12)
    plan.fft_c2r(d)
    assert float((d[:, :, :ng] / ng ** 3 - x).norm() / x.norm()) < 1e-13


@pytest.mark.parametrize("ng", [16, 48, 64, 96, 1024])
def test_fft_f32(pmpkg, ng):
    rng = np.random.default_rng(3)
    m = np.zeros((ng, ng, ng + 2), np.float32)
    m[:, :, :ng] = rng.standard_normal((ng, ng, ng)).astype(np.float32)
    plan = pmpkg.Plan(ng, "fp32")
    d = T(m, torch.float32)
    plan.fft_r2c(d)
    if ng <= 96:
        assert rel(H(d).view(np.complex64), np.fft.rfftn(m[:, :, :ng].astype(np.float64))) < 2e-6
    plan.fft_c2r(d)
    assert rel(H(d)[:, :, :ng] / ng ** 3, m[:, :, :ng]) < 2e-6


@pytest.mark.parametrize("kind", ["discrete", "spectral"])
@pytest.mark.parametrize("ng", [512, 1024])
def test_fft_and_poisson_f32_large_match_f64(pmpkg, ng, kind):
    """Meshes larger than L2 (the pipelined persistent strided passes): the
    FP32 spectrum and the FP32 fused Poisson solve against the FP64 plan."""
    g = torch.Generator(device=DEV).manual_seed(ng + 7)
    x = torch.randn((ng, ng, ng), generator=g, device=DEV, dtype=torch.float64)
    p64, p32 = pmpkg.Plan(ng, "fp64", kind), pmpkg.Plan(ng, "fp32", kind)
    d64, d32 = p64.new_mesh(), p32.new_mesh()
    d64[:, :, :ng] = x
    d32[:, :, :ng] = x.float()
    p64.fft_r2c(d64)
    p32.fft_r2c(d32)
    err = float((d32.double() - d64).norm() / d64.norm())
    assert err < 2e-6, err
    d64[:, :, :ng], d32[:, :, :ng] = x, x.float()
    d64[:, :, ng:], d32[:, :, ng:] = 0, 0
    p64.poisson(d64, 2.5)
    p32.poisson(d32, 2.5)
    err = float((d32[:, :, :ng].double() - d64[:, :, :ng]).norm() / d64[:, :, :ng].norm())
    assert err < 2e-6, err
    del d64, d32, x
    torch.cuda.empty_cache()


@pytest.mark.parametrize("ng", [64, 512])
def test_fft_f32_cross_checks_against_cufft(pmpkg, ng):
    """The hand-written FP32 R2C against cuFFT (torch.fft.rfftn on the GPU),
    cuFFT only as an independent cross-check: relative L2 < 2e-6."""
    g = torch.Generator(device=DEV).manual_seed(ng + 3)
    x = torch.randn((ng, ng, ng), generator=g, device=DEV, dtype=torch.float32)
    plan = pmpkg.Plan(ng, "fp32")
    d = plan.new_mesh()
    d[:, :, :ng] = x
    plan.fft_r2c(d)
    ours = torch.view_as_complex(d.view(ng, ng, ng // 2 + 1, 2))
    ref = torch.fft.rfftn(x.double())
    err = float((ours.to(torch.complex128) - ref).abs().norm() / ref.abs().norm())
    assert err < 2e-6, err
    del d, x, ours, ref
    torch.cuda.empty_cache()


@pytest.mark.parametrize("kind", ["discrete", "spectral"])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_green_and_fused_poisson(pmpkg, O, kind, prec):
    ng = 32
    rng = np.random.default_rng(11)
    m = O.padded(ng)
    m[:, :, :ng] = rng.standard_normal((ng, ng, ng))
    kid = 0 if kind == "discrete" else 1
    ref = m.copy()
    O.rfft3d_forward(ref)
    O.green(ref, 2.5, kid)
    spec_ref = O.spectrum_view(ref).copy()
    O.rfft3d_inverse(ref)
    dt = torch.float64 if prec == "fp64" else torch.float32
    tol = 1e-12 if prec == "fp64" else 2e-6
    plan = pmpkg.Plan(ng, prec, kind)
    d = T(m, dt)
    plan.fft_r2c(d)
    plan.green(d, 2.5)
    got = H(d).astype(np.float64) if prec == "fp32" else H(d)
    assert rel(got.view(np.complex128), spec_ref) < tol
    plan.fft_c2r(d)
    assert rel(H(d)[:, :, :ng], ref[:, :, :ng]) < tol
    e = T(m, dt)
    plan.poisson(e, 2.5)
    assert rel(H(e)[:, :, :ng], ref[:, :, :ng]) < tol


# ------------------------------------------------------ particle stages

@pytest.mark.parametrize("ng,np_", [(8, 100), (16, 5000), (64, 64 ** 3)])
def test_deposit_f64(pmpkg, O, ng, np_):
    x, y, z = uniform(ng, np_, ng)
    mass = ng ** 3 / np_
    plan = pmpkg.Plan(ng, "fp64")
    got = H(plan.deposit(T(x), T(y), T(z), mass))
    ref = O.deposit(ng, x, y, z, mass)
    assert rel(got, ref) < 1e-13
    assert np.all(got[:, :, ng:] == 0)


@pytest.mark.parametrize("order", [2, 4])
def test_gradient_f64(pmpkg, O, order):
    ng = 32
    rng = np.random.default_rng(order)
    phi = O.padded(ng)
    phi[:, :, :ng] = rng.standard_normal((ng, ng, ng))
    plan = pmpkg.Plan(ng, "fp64", grad_order=order)
    f = plan.gradient(T(phi))
    ref = O.gradient(phi, order)
    for a in range(3):
        assert rel(H(f[a]), ref[a]) < 1e-14


def test_interp_kick_and_drift_f64(pmpkg, O):
    ng, np_ = 32, 20000
    x, y, z = uniform(ng, np_, 5)
    rng = np.random.default_rng(6)
    f = [rng.standard_normal((ng, ng, ng)) for _ in range(3)]
    p = [rng.standard_normal(np_) for _ in range(3)]
    plan = pmpkg.Plan(ng, "fp64")
    tp = [T(a) for a in p]
    tx = [T(a) for a in (x, y, z)]
    plan.interp_kick(*tx, [T(a) for a in f], *tp, 0.37)
    O.interp_kick(x, y, z, f, *p, 0.37)
    for a in range(3):
        assert rel(H(tp[a]), p[a]) < 1e-14
    plan.drift(*tx, *tp, 3.1)
    O.drift(ng, x, y, z, *p, 3.1)
    for a, b in zip(tx, (x, y, z)):
        assert np.abs(H(a) - b).max() < 1e-12
        assert H(a).min() >= 0 and H(a).max() < ng


# --------------------------------------- whole reference step vs golden

@pytest.mark.parametrize("name", golden_cases())
def test_reference_step_matches_golden(pmpkg, name):
    g = load_golden(name)
    ng, mass = int(g["ng"]), float(g["mass"])
    cp, ck = pmpkg.reference_coefficients(float(g["a"]))
    plan = pmpkg.Plan(ng, "fp64")
    x, y, z = (T(g["pos"][i]) for i in range(3))
    p = [torch.zeros_like(x) for _ in range(3)]
    mesh = plan.deposit(x, y, z, mass)
    assert rel(H(mesh)[:, :, :ng], g["delta"]) < 1e-13
    plan.fft_r2c(mesh)
    plan.green(mesh, cp)
    plan.fft_c2r(mesh)
    if "phi" in g:
        assert rel(H(mesh)[:, :, :ng], g["phi"]) < 1e-12
    f = plan.gradient(mesh)
    if "force" in g:
        assert rel(np.stack([H(a) for a in f]), g["force"]) < 1e-12
    plan.interp_kick(x, y, z, f, *p, ck)
    assert rel(np.stack([H(a) for a in p]), g["mom"]) < 1e-12
    # the one-call step gives the same momenta
    q = [torch.zeros_like(x) for _ in range(3)]
    plan.step(x, y, z, *q, mass, cp, ck, 0.0)
    assert rel(np.stack([H(a) for a in q]), g["mom"]) < 1e-12


def test_reference_mirrors(pmpkg):
    """The reference-named functions reproduce the golden step."""
    g = load_golden("ref_step_ng16_np16.npz")
    ng = int(g["ng"])
    x, y, z = (T(g["pos"][i]) for i in range(3))
    buf = torch.zeros((ng, ng, ng + 2), dtype=torch.float64, device=DEV)
    pmpkg.deposit_particles(x, y, z, buf, float(g["mass"]))
    fft = pmpkg.FFT(ng, buf)
    fft.forward()
    fft.apply_green(float(g["a"]))
    fft.backward()
    d = [torch.empty((ng, ng, ng), dtype=torch.float64, device=DEV) for _ in range(3)]
    pmpkg.centered_derivatives(buf, *d)
    p = [torch.zeros_like(x) for _ in range(3)]
    pmpkg.update_particles(x, y, z, *d, *p, float(g["a"]))
    assert rel(np.stack([H(a) for a in p]), g["mom"]) < 1e-12


@pytest.mark.parametrize("ng,nrow,kind,order", [(64, 64, "discrete", 2), (128, 64, "spectral", 4),
                                                (256, 256, "discrete", 2)])
def test_full_step_f64_vs_oracle(pmpkg, O, ng, nrow, kind, order):
    x, y, z = uniform(ng, nrow ** 3, ng + nrow)
    mass = ng ** 3 / nrow ** 3
    cp, ck = 4 * np.pi, 0.01
    kid = 0 if kind == "discrete" else 1
    p = [np.zeros(nrow ** 3) for _ in range(3)]
    delta, phi, f = O.force_step(ng, x, y, z, *p, mass, cp, ck, kid, order)
    plan = pmpkg.Plan(ng, "fp64", kind, order)
    tx = [T(a) for a in (x, y, z)]
    tp = [torch.zeros_like(tx[0]) for _ in range(3)]
    plan.step(*tx, *tp, mass, cp, ck, 0.0)
    phi_g = H(plan.workspace_mesh())
    assert rel(phi_g[:, :, :ng], phi[:, :, :ng]) < 1e-12
    assert rel(np.stack([H(a) for a in tp]), np.stack(p)) < 1e-12


# ------------------------------------------------------------- FP32 split

def test_split_join(pmpkg, O):
    ng, np_ = 64, 100000
    x, y, z = uniform(ng, np_, 2)
    x[:3] = [0.0, ng - 1e-12, 5.0 - 1e-17]
    plan = pmpkg.Plan(ng, "fp32")
    cell, off = plan.split(T(x), T(y), T(z))
    ocell, ooff = O.split_positions(ng, x, y, z)
    back = plan.join(cell, off)
    for a, b in zip(back, (x, y, z)):
        d = np.abs(H(a) - b)
        d = np.minimum(d, ng - d)
        assert d.max() <= 2 ** -24
    assert np.all(H(off[0]) < 1.0) and np.all(H(off[0]) >= 0.0)


@pytest.mark.parametrize("ng,nrow,kind,order", [(64, 64, "discrete", 2), (64, 32, "spectral", 4),
                                                (128, 64, "spectral", 4), (48, 48, "spectral", 4),
                                                (96, 96, "discrete", 2)])
def test_split_forces_within_1e4_of_fp64(pmpkg, O, ng, nrow, kind, order):
    pos, vel = O.zeldovich_ic(ng, nrow, -2.0, 0.5, seed=ng + nrow)
    mass = ng ** 3 / nrow ** 3
    cp = 4 * np.pi
    kid = 0 if kind == "discrete" else 1
    fr = [np.zeros(nrow ** 3) for _ in range(3)]
    delta, phi, f = O.force_step(ng, *pos, *fr, mass, cp, 1.0, kid, order)
    plan = pmpkg.Plan(ng, "fp32", kind, order)
    cell, off = plan.split(*(T(a) for a in pos))
    mesh = plan.deposit_split(cell, off, mass)
    assert rel(H(mesh)[:, :, :ng], delta[:, :, :ng]) < 1e-6
    plan.poisson(mesh, cp)
    assert rel(H(mesh)[:, :, :ng], phi[:, :, :ng]) < 1e-4
    g = plan.interp_split(mesh, cell, off)
    err = rel(np.stack([H(a) for a in g]), np.stack(fr))
    assert err < 1e-4, err


@pytest.mark.parametrize("ng,np_,mode", [(8, 300, "uniform"), (16, 4096, "faces"), (32, 40000, "uniform"),
                                         (64, 0, "uniform"), (128, 300000, "faces")])
def test_tile_deposit_f32_matches_oracle(pmpkg, O, ng, np_, mode):
    """Binned owner-computes deposit, including particles on tile faces,
    edges and the periodic wrap, and an empty particle set."""
    rng = np.random.default_rng(ng + np_)
    pos = [rng.uniform(0, ng, np_) for _ in range(3)]
    if mode == "faces" and np_:
        ts = 16 if ng >= 16 else 8
        for a in range(3):  # a third of the particles in the last cell of a tile, some at ng - 1
            sel = rng.random(np_) < 0.34
            pos[a][sel] = (rng.integers(0, ng // ts, sel.sum()) * ts + ts - 1) + rng.random(sel.sum())
    mass = 1.7
    plan = pmpkg.Plan(ng, "fp32")
    cell, off = plan.split(*(T(a) for a in pos))
    got = H(plan.deposit_split(cell, off, mass)).astype(np.float64)
    x, y, z = (H(a) for a in plan.join(cell, off))
    ref = O.deposit(ng, x, y, z, mass)
    assert np.abs(got - ref).max() < 1e-5 * max(1.0, mass * np_ / ng ** 3 * 8)
    assert np.all(got[:, :, ng:] == 0)


def test_sort_preserves_particles_and_step(pmpkg, O):
    ng, nrow = 64, 32
    pos, vel = O.zeldovich_ic(ng, nrow, -2.0, 0.5, seed=9)
    plan = pmpkg.Plan(ng, "fp32", "spectral", 4)
    cell, off = plan.split(*(T(a) for a in pos))
    v = [T(a, torch.float32) for a in vel]
    before = np.stack([H(cell).astype(np.float64)] + [H(a) for a in off] + [H(a) for a in v])
    m0 = H(plan.deposit_split(cell, off, 1.0))
    plan.sort_split(cell, off, v)
    after = np.stack([H(cell).astype(np.float64)] + [H(a) for a in off] + [H(a) for a in v])
    order_b = np.lexsort(before[::-1])
    order_a = np.lexsort(after[::-1])
    assert np.array_equal(before[:, order_b], after[:, order_a])  # same particles
    assert not np.array_equal(before, after)                      # in a new order
    tiles = (H(cell) >> 24, (H(cell) >> 14) & 63, (H(cell) >> 4) & 63)
    assert len(np.unique(np.stack(tiles), axis=1).T) > 1
    m1 = H(plan.deposit_split(cell, off, 1.0))
    assert np.abs(m1 - m0).max() < 1e-5


@pytest.mark.parametrize("ng,nrow", [(32, 32), (128, 64), (256, 128), (512, 64), (1024, 128)])
def test_fused_step_matches_stagewise(pmpkg, O, ng, nrow):
    """pm_step_f32 (deposit fused with the z FFT pass) equals the separate
    stages deposit -> Poisson -> kick + drift on the same state."""
    pos, vel = O.zeldovich_ic(ng, nrow, -1.5, 1.0, seed=ng)
    mass, cp, dt = ng ** 3 / nrow ** 3, 4 * np.pi, 0.01
    plan = pmpkg.Plan(ng, "fp32", "spectral", 4)
    cell, off = plan.split(*(T(a) for a in pos))
    v = [T(a, torch.float32) for a in vel]
    c1, o1, v1 = cell.clone(), [t.clone() for t in off], [t.clone() for t in v]
    plan.step_split(c1, o1, v1, mass, cp, dt, dt)
    mesh = plan.deposit_split(cell, off, mass)
    plan.poisson(mesh, cp)
    plan.kick_drift_split(mesh, cell, off, v, dt, dt)
    phi_fused = plan.workspace_mesh()[:, :, :ng]
    err = float((phi_fused.double() - mesh[:, :, :ng].double()).norm() / mesh[:, :, :ng].double().norm())
    assert err < 1e-6, err
    # velocities: the kick amplifies the potential's FP32 rounding differences
    # (summation order of the two deposits) through the 4-point gradient; at
    # ng = 1024 with 128^3 particles (mass 512 each) they reach ~1.3e-6
    assert rel(np.stack([H(a) for a in v1]), np.stack([H(a) for a in v])) < (1e-6 if ng < 1024 else 3e-6)
    del mesh, phi_fused
    plan.close()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_conserved_reductions(pmpkg, O, prec):
    """pm_reduce_*: the FP64 mesh total equals the deposited mass, the
    momentum equals mass * sum(v) in FP64, repeated calls give identical bits,
    and a few KDK steps conserve momentum (CIC deposit and interpolation with
    a centred difference exert no net force)."""
    ng, nrow = 64, 32
    pos, vel = O.zeldovich_ic(ng, nrow, -2.0, 0.7, seed=5)
    mass, cp, dt = ng ** 3 / nrow ** 3, 4 * np.pi, 0.05
    plan = pmpkg.Plan(ng, prec, "spectral", 4)
    dt_ = torch.float64 if prec == "fp64" else torch.float32
    v = [T(a, dt_) for a in vel]
    if prec == "fp64":
        x = [T(a) for a in pos]
        mesh = plan.deposit(*x, mass)
        step = lambda: plan.step(*x, *v, mass, cp, dt, dt)  # noqa: E731
    else:
        cell, off = plan.split(*(T(a) for a in pos))
        mesh = plan.deposit_split(cell, off, mass)
        step = lambda: plan.step_split(cell, off, v, mass, cp, dt, dt)  # noqa: E731
    c1 = plan.conserved(mesh, v, mass)
    c2 = plan.conserved(mesh, v, mass)
    assert c1 == c2
    total = mass * nrow ** 3
    assert abs(c1["mass"] - total) / total < (1e-12 if prec == "fp64" else 1e-5)
    ref = [mass * float(t.double().sum()) for t in v]
    scale = mass * float(sum(t.double().abs().sum() for t in v))
    assert max(abs(a - b) for a, b in zip(c1["momentum"], ref)) < 1e-12 * scale
    for _ in range(5):
        step()
    c3 = plan.conserved(None, v, mass)
    assert c3["mass"] == 0.0
    drift = max(abs(a - b) for a, b in zip(c3["momentum"], c1["momentum"]))
    assert drift < (1e-9 if prec == "fp64" else 1e-5) * scale, drift / scale


@pytest.mark.parametrize("ng", [32, 48])
def test_split_kernels_wrap_out_of_range_cells(pmpkg, O, ng):
    """A cell word whose indices lie outside [0, ng) (here i + ng, j + 2 ng)
    is the same periodic cell: the FP32 kernels wrap it before any mesh
    access, so interpolation, deposit and the adjoint gather give the same
    results as for the canonical word."""
    nrow = 16
    pos, _ = O.zeldovich_ic(ng, nrow, -2.0, 0.5, seed=21)
    plan = pmpkg.Plan(ng, "fp32", "spectral", 4)
    cell, off = plan.split(*(T(a) for a in pos))
    bad = cell.clone()
    sel = torch.arange(cell.numel(), device=DEV) % 3 == 0
    bad[sel] = bad[sel] + (ng << 20) + ((2 * ng) << 10)
    mass, cp = ng ** 3 / nrow ** 3, 4 * np.pi
    phi = plan.poisson(plan.deposit_split(cell, off, mass), cp)
    assert rel(H(plan.deposit_split(bad, off, mass)), H(plan.deposit_split(cell, off, mass))) < 1e-6
    f0, f1 = plan.interp_split(phi, cell, off), plan.interp_split(phi, bad, off)
    assert all(torch.equal(a, b) for a, b in zip(f0, f1))
    dbar = torch.randn((ng, ng, ng + 2), dtype=torch.float32, device=DEV)
    b0 = [torch.zeros_like(off[0]) for _ in range(3)]
    b1 = [torch.zeros_like(off[0]) for _ in range(3)]
    plan.adjoint_deposit_split(cell, off, mass, dbar, b0)
    plan.adjoint_deposit_split(bad, off, mass, dbar, b1)
    assert all(torch.equal(a, b) for a, b in zip(b0, b1))


def test_split_run_tracks_fp64_over_50_kdk_steps(pmpkg, O):
    """The mixed-precision configuration in miniature (128^3 particles on a
    256^3 mesh, P(k) ~ k^-1.5, rms 1 cell, 50 KDK steps at dt = 0.005): final
    positions of the FP32 split path within 1e-4 cells of the FP64 path run
    from the same state, the final density within 1e-4 relative L2."""
    ng, nrow, steps, dt = 256, 128, 50, 0.005
    pos, vel = O.zeldovich_ic(ng, nrow, -1.5, 1.0, seed=77)
    mass, cp = ng ** 3 / nrow ** 3, 4 * np.pi
    p64, p32 = pmpkg.Plan(ng, "fp64", "spectral", 4), pmpkg.Plan(ng, "fp32", "spectral", 4)
    x = [T(a) for a in pos]
    v = [T(a) for a in vel]
    cell, off = p32.split(*x)
    w = [T(a, torch.float32) for a in vel]
    for s in range(steps + 1):
        ck, dd = (0.5 * dt if s in (0, steps) else dt), (dt if s < steps else 0.0)
        p64.step(*x, *v, mass, cp, ck, dd)
        p32.step_split(cell, off, w, mass, cp, ck, dd)
    j = p32.join(cell, off)
    dmax = 0.0
    for a, b in zip(j, x):
        d = torch.remainder(a - b + 0.5 * ng, float(ng)) - 0.5 * ng
        dmax = max(dmax, float(d.abs().max()))
    assert dmax < 1e-4, dmax
    d32 = p32.deposit_split(cell, off, mass)[:, :, :ng].double()
    d64 = p64.deposit(*x, mass)[:, :, :ng]
    assert float((d32 - d64).norm() / (d64 + 1.0).norm()) < 1e-4


def test_stage_timers_count_every_kernel_of_a_step(pmpkg, O):
    """The stage timers that bench.py's gpu_launches comes from count each
    kernel launch of pm_step_f32: binning (count, three scans, scatter), the
    fused deposit, y / x + Green / y passes, z C2R and the gather: 11."""
    ng, nrow = 64, 32
    pos, vel = O.zeldovich_ic(ng, nrow, -2.0, 0.5, seed=9)
    plan = pmpkg.Plan(ng, "fp32", "spectral", 4)
    cell, off = plan.split(*(T(a) for a in pos))
    v = [T(a, torch.float32) for a in vel]
    plan.read_timing(reset=True)
    plan.set_timing(True)
    plan.step_split(cell, off, v, ng ** 3 / nrow ** 3, 4 * np.pi, 0.01, 0.01)
    t = plan.read_timing(reset=True)
    plan.set_timing(False)
    n = {k: c for k, (_, c) in t.items()}
    assert n == {"bin": 5, "deposit": 1, "fft_y_fwd": 1, "fft_x_green": 1, "fft_y_inv": 1, "fft_z_c2r": 1,
                 "kick_drift": 1}, n
    assert all(ms > 0 for ms, _ in t.values())


@pytest.mark.parametrize("ng", [48, 64])
def test_empty_particle_set_through_every_step(pmpkg, ng):
    """np = 0: the FP64 and FP32 steps (fused deposit at 64, tile deposit at
    48), the adjoints and the reductions run without error; the density is
    the uniform -1 background, so the potential vanishes."""
    e64 = [torch.zeros(0, dtype=torch.float64, device=DEV) for _ in range(6)]
    e32 = [torch.zeros(0, dtype=torch.float32, device=DEV) for _ in range(6)]
    ecell = torch.zeros(0, dtype=torch.int32, device=DEV)
    p32 = pmpkg.Plan(ng, "fp32", "spectral", 4)
    p32.step_split(ecell, e32[:3], e32[3:], 1.0, 4 * np.pi, 0.01, 0.01)
    assert float(p32.workspace_mesh()[:, :, :ng].abs().max()) < 1e-6
    p32.step_adjoint_split(ecell, e32[:3], 1.0, 4 * np.pi, 0.01, 0.01, e32[:3], e32[3:])
    m = p32.deposit_split(ecell, e32[:3], 1.0)
    assert torch.all(m[:, :, :ng] == -1.0)
    c = p32.conserved(m, e32[3:], 1.0)
    assert c["mass"] == 0.0 and c["momentum"] == [0.0, 0.0, 0.0]
    if ng & (ng - 1) == 0:
        p64 = pmpkg.Plan(ng, "fp64", "spectral", 4)
        p64.step(*e64, 1.0, 4 * np.pi, 0.01, 0.01)
        assert float(p64.workspace_mesh()[:, :, :ng].abs().max()) < 1e-12
        p64.step_adjoint(*e64[:3], 1.0, 4 * np.pi, 0.01, 0.01, e64[:3], e64[3:])
    p32.check()


def test_fp32_paths_reject_more_than_2_32_particles(pmpkg):
    """The FP32 binning indexes particles with 32 bits: a count of 2^32 is
    refused with PM_ERR_SIZE before any kernel runs (the small arrays passed
    here are never read)."""
    import ctypes
    plan = pmpkg.Plan(64, "fp32")
    a = [torch.zeros(16, dtype=torch.float32, device=DEV) for _ in range(7)]
    c = torch.zeros(16, dtype=torch.int32, device=DEV)
    mesh = plan.new_mesh()
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    big = 1 << 32
    rc = plan.lib.pm_deposit_f32(plan.handle, vp(c), vp(a[0]), vp(a[1]), vp(a[2]), big, 1.0, vp(mesh))
    assert rc == 2 and b"2^32" in plan.lib.pm_last_error()
    rc = plan.lib.pm_step_f32(plan.handle, vp(c), *(vp(t) for t in a[:6]), big, 1.0, 1.0, 0.01, 0.01)
    assert rc == 2
    torch.cuda.synchronize()


def test_split_step_kick_drift(pmpkg, O):
    ng, nrow = 64, 32
    pos, vel = O.zeldovich_ic(ng, nrow, -2.0, 0.5, seed=3)
    mass = ng ** 3 / nrow ** 3
    cp, dt = 4 * np.pi, 0.5
    # oracle: force at x, v += f dt, x += v dt
    x, y, z = (a.copy() for a in pos)
    v = [a.copy() for a in vel]
    O.force_step(ng, x, y, z, *v, mass, cp, dt, 1, 4)
    O.drift(ng, x, y, z, *v, dt)
    plan = pmpkg.Plan(ng, "fp32", "spectral", 4)
    cell, off = plan.split(*(T(a) for a in pos))
    tv = [T(a, torch.float32) for a in vel]
    plan.step_split(cell, off, tv, mass, cp, dt, dt)
    assert rel(np.stack([H(a) for a in tv]), np.stack(v)) < 1e-5
    got = plan.join(cell, off)
    for a, b in zip(got, (x, y, z)):
        d = np.abs(H(a) - b)
        d = np.minimum(d, ng - d)
        assert d.max() < 1e-4


# ---------------------------------------------------- initial conditions

@pytest.mark.parametrize("ng,nrow,ns,rms", [(16, 16, -2.0, 0.3), (64, 32, -1.5, 1.0), (48, 48, -2.5, 0.7)])
def test_zeldovich_ic_matches_oracle(pmpkg, O, ng, nrow, ns, rms):
    pos, vel = pmpkg.zeldovich_ic(ng, nrow, ns, rms, seed=42, device=DEV)
    opos, ovel = O.zeldovich_ic(ng, nrow, ns, rms, seed=42)
    assert rel(np.stack([H(a) for a in vel]), np.stack(ovel)) < 1e-12
    for a, b in zip(pos, opos):
        d = np.abs(H(a) - b)
        d = np.minimum(d, ng - d)
        assert d.max() < 1e-11


def test_kdk_run_f64_matches_oracle(pmpkg, O):
    """10 KDK steps (spectral Poisson, 4-point gradient), 32^3 on 32^3."""
    ng = nrow = 32
    pos, vel = O.zeldovich_ic(ng, nrow, -2.0, 0.3, seed=1)
    cp, dt, steps = 4 * np.pi, 0.01, 10
    x, y, z = (a.copy() for a in pos)
    v = [a.copy() for a in vel]
    O.kdk(ng, x, y, z, *v, 1.0, cp, dt, steps, 1, 4)
    plan = pmpkg.Plan(ng, "fp64", "spectral", 4)
    tx = [T(a) for a in pos]
    tv = [T(a) for a in vel]
    for s in range(steps + 1):
        ck = 0.5 * dt if s in (0, steps) else dt
        plan.step(*tx, *tv, 1.0, cp, ck, dt if s < steps else 0.0)
    assert rel(np.stack([H(a) for a in tv]), np.stack(v)) < 1e-11
    for a, b in zip(tx, (x, y, z)):
        d = np.abs(H(a) - b)
        assert np.minimum(d, ng - d).max() < 1e-11


# --------------------------------------------------------------- errors

def test_errors_are_reported(pmpkg):
    plan = pmpkg.Plan(16, "fp64")
    x = torch.full((4,), 3.0, dtype=torch.float64, device=DEV)
    x[1] = float("nan")
    x[2] = 17.5
    y = torch.ones_like(x)
    z = torch.ones_like(x)
    plan.deposit(x, y, z, 1.0)
    with pytest.raises(pmpkg.PMError) as e:
        plan.check()
    assert e.value.code == 5  # PM_ERR_RANGE
    plan.check()  # flag was cleared
    with pytest.raises(pmpkg.PMError) as e:
        pmpkg.Plan(12, "fp64")
    assert e.value.code == 2  # PM_ERR_SIZE
    with pytest.raises(pmpkg.PMError) as e:
        pmpkg.Plan(36, "fp64")  # 36 = 4 x 9: not a supported mixed-radix size
    assert e.value.code == 2
    p32 = pmpkg.Plan(16, "fp32")
    with pytest.raises(pmpkg.PMError):
        p32.deposit(x, y, z, 1.0)  # FP64 entry point on an FP32 plan
    with pytest.raises(pmpkg.PMError):
        plan.deposit(x.float(), y, z, 1.0)


@pytest.mark.parametrize("ng", [256, 512])
def test_poisson_f32_transposed_spectrum(pmpkg, ng):
    """FP32 plans of ng >= 512 route the x + Green pass through a second half
    spectrum laid out [ky][kx][kz]: the first pm_poisson_f32 adds exactly
    ng^2 (ng/2+1) complex64 to the plan's device bytes (nothing for smaller
    meshes, which solve in place), later solves add nothing, and solving the
    same mesh twice gives the same bits."""
    g = torch.Generator(device=DEV).manual_seed(ng + 11)
    plan = pmpkg.Plan(ng, "fp32")
    d = plan.new_mesh()
    d[:, :, :ng] = torch.randn((ng, ng, ng), generator=g, device=DEV, dtype=torch.float32)
    x = d.clone()
    b0 = plan.device_bytes()
    plan.poisson(d, 2.5)
    grown = plan.device_bytes() - b0
    assert grown == (ng * ng * (ng // 2 + 1) * 8 if ng >= 512 else 0)
    e = x.clone()
    plan.poisson(e, 2.5)
    assert plan.device_bytes() - b0 == grown
    assert torch.equal(d, e)
    del d, e, x
    torch.cuda.empty_cache()


@pytest.mark.parametrize("ng,nrow", [(256, 128), (512, 128)])
def test_tiled_gather_matches_cached(pmpkg, O, ng, nrow):
    """pm_step_f32 with the shared-memory tiled gather (bin order by column
    tile, class and z chunk) against the default cached gather on the same
    state, the particles in Lagrangian and in shuffled order: velocities
    within 2e-6 relative L2 (the two deposits' binnings sum in different
    orders), positions within 1e-5 cells."""
    pos, vel = O.zeldovich_ic(ng, nrow, -1.5, 1.0, seed=ng + 1)
    mass, cp, dt = ng ** 3 / nrow ** 3, 4 * np.pi, 0.01
    ref = pmpkg.Plan(ng, "fp32", "spectral", 4)
    tiled = pmpkg.Plan(ng, "fp32", "spectral", 4)
    tiled.set_gather("tiled")
    cell, off = ref.split(*(T(a) for a in pos))
    v = [T(a, torch.float32) for a in vel]
    shuffle = torch.randperm(nrow ** 3, generator=torch.Generator().manual_seed(3)).to(DEV)
    for order in (None, shuffle):
        sel = (lambda t: t) if order is None else (lambda t: t[order].contiguous())
        c0, o0, v0 = sel(cell), [sel(a) for a in off], [sel(a) for a in v]
        c1, o1, v1 = c0.clone(), [a.clone() for a in o0], [a.clone() for a in v0]
        ref.step_split(c0, o0, v0, mass, cp, dt, dt)
        tiled.step_split(c1, o1, v1, mass, cp, dt, dt)
        tiled.check()
        err = rel(np.stack([H(a) for a in v1]), np.stack([H(a) for a in v0]))
        assert err < 2e-6, err
        x0, x1 = ref.join(c0, o0), ref.join(c1, o1)
        d = max(float((torch.remainder(a - b + ng / 2, ng) - ng / 2).abs().max()) for a, b in zip(x1, x0))
        assert d < 1e-5, d
    with pytest.raises(pmpkg.PMError):
        pmpkg.Plan(128, "fp32").set_gather("tiled")  # below 256 cells: PM_ERR_SIZE


@pytest.mark.parametrize("ng,nrow", [(64, 32), (1024, 64)])
def test_potential_then_ranged_kick_drift_equals_step(pmpkg, O, ng, nrow):
    """pm_potential_f32 followed by pm_kick_drift_f32: over four particle
    ranges it gives the whole-range gather's state bit for bit (the gather is
    per particle), and the pair gives pm_step_f32's state within FP32
    rounding (the deposit's shared-memory atomics sum in no fixed order)."""
    pos, vel = O.zeldovich_ic(ng, nrow, -1.5, 1.0, seed=ng + 7)
    mass, cp, dt = ng ** 3 / nrow ** 3, 4 * np.pi, 0.01
    plan = pmpkg.Plan(ng, "fp32", "spectral", 4)
    cell, off = plan.split(*(T(a) for a in pos))
    v = [T(a, torch.float32) for a in vel]
    c1, o1, v1 = cell.clone(), [a.clone() for a in off], [a.clone() for a in v]
    c2, o2, v2 = cell.clone(), [a.clone() for a in off], [a.clone() for a in v]
    plan.step_split(cell, off, v, mass, cp, dt, dt)
    phi = plan.potential_split(c1, o1, mass, cp)
    plan.kick_drift_split(phi, c2, o2, v2, dt, dt)
    n = nrow ** 3
    for lo, hi in ((0, n // 3), (n // 3, n // 2), (n // 2, n - 5), (n - 5, n)):
        plan.kick_drift_split(phi, c1[lo:hi], [a[lo:hi] for a in o1], [a[lo:hi] for a in v1], dt, dt)
    plan.check()
    assert torch.equal(c1, c2)
    for a, b in zip(o1 + v1, o2 + v2):
        assert torch.equal(a, b)
    err = rel(np.stack([H(a) for a in v1]), np.stack([H(a) for a in v]))
    assert err < 1e-6, err
    x0, x1 = plan.join(cell, off), plan.join(c1, o1)
    d = max(float((torch.remainder(a - b + ng / 2, ng) - ng / 2).abs().max()) for a, b in zip(x1, x0))
    assert d < 1e-5, d
    plan.close()
