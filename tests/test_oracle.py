"""The CPU oracle, pinned against the reference.

* every golden fixture (made by tests/golden/make_golden.py from the
  reference's own compiled kernels) against the restatement;
* the restatement against the reference compiled here (oracle/_ref), when
  the reference sources were available to build it;
* the oracle FFT against numpy.fft;
* known-answer tests of the step (single particle, uniform lattice, single
  Fourier mode, momentum conservation, R2C/C2R round trip).
"""
import numpy as np
import pytest

from conftest import golden_cases, load_golden


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


@pytest.mark.parametrize("n", [2, 3, 4, 5, 6, 8, 12, 16, 30, 48, 64, 96, 128])
def test_fft1d_matches_numpy(O, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert rel(O.fft1d(a, -1), np.fft.fft(a)) < 1e-14
    assert rel(O.fft1d(a, +1), np.fft.ifft(a) * n) < 1e-14


@pytest.mark.parametrize("ng", [8, 16, 32])
def test_rfft3d_matches_numpy_and_round_trips(O, ng):
    rng = np.random.default_rng(ng)
    m = O.padded(ng)
    m[:, :, :ng] = rng.standard_normal((ng, ng, ng))
    x = m[:, :, :ng].copy()
    O.rfft3d_forward(m)
    assert rel(O.spectrum_view(m), np.fft.rfftn(x)) < 1e-14
    O.rfft3d_inverse(m)
    # unnormalised pair: C2R(R2C(x)) = ng^3 x (FFTW convention)
    assert rel(m[:, :, :ng], ng ** 3 * x) < 1e-14


@pytest.mark.parametrize("name", golden_cases())
def test_restatement_matches_golden(O, name):
    g = load_golden(name)
    ng, mass = int(g["ng"]), float(g["mass"])
    x, y, z = (np.ascontiguousarray(g["pos"][i]) for i in range(3))
    px, py, pz = (np.zeros_like(x) for _ in range(3))
    cp, ck = O.reference_coefficients(float(g["a"]))
    delta, phi, f = O.force_step(ng, x, y, z, px, py, pz, mass, cp, ck, green_kind=0, grad_order=2)
    assert rel(delta[:, :, :ng], g["delta"]) < 1e-13
    if "phi" in g:
        assert rel(phi[:, :, :ng], g["phi"]) < 1e-12
        assert rel(np.stack(f), g["force"]) < 1e-12
    assert rel(np.stack([px, py, pz]), g["mom"]) < 1e-12


@pytest.mark.parametrize("ng,nrow", [(8, 8), (16, 16), (16, 8), (32, 32)])
def test_restatement_matches_compiled_reference(O, ng, nrow):
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    x, y, z = O.reference_init_particles(ng, nrow)
    mass = ng ** 3 / nrow ** 3
    px, py, pz = (np.zeros(nrow ** 3) for _ in range(3))
    r = O.reference_force_step(ng, x, y, z, px, py, pz, mass, threads=3)
    qx, qy, qz = (np.zeros(nrow ** 3) for _ in range(3))
    cp, ck = O.reference_coefficients()
    d, phi, f = O.force_step(ng, x, y, z, qx, qy, qz, mass, cp, ck)
    assert rel(d[:, :, :ng], r["delta"][:, :, :ng]) < 1e-13
    assert rel(phi[:, :, :ng], r["phi"][:, :, :ng]) < 1e-12
    for a in range(3):
        assert rel(f[a], r["forces"][a][:ng, :ng, :ng]) < 1e-12
        # the reference's + ghost plane of the force is the periodic image
        assert np.array_equal(r["forces"][a][ng, :ng, :ng], r["forces"][a][0, :ng, :ng])
    assert rel(np.stack([qx, qy, qz]), np.stack([px, py, pz])) < 1e-12


def test_golden_fixtures_reproduce(O):
    """The committed fixtures are what the compiled reference produces now."""
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    import importlib.util
    import os
    from conftest import ROOT
    spec = importlib.util.spec_from_file_location("mg", os.path.join(ROOT, "tests", "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    for ng, nrow in mg.CASES:
        d = mg.make(ng, nrow, full=ng <= 16)
        g = load_golden(f"ref_step_ng{ng}_np{nrow}.npz")
        for k in d:
            assert np.allclose(d[k], g[k], rtol=1e-13, atol=1e-15), k


# ------------------------------------------------------------ known answers

def test_single_particle_on_lattice_point(O):
    ng = 8
    x, y, z = (np.array([v]) for v in (3.0, 5.0, 7.0))
    m = O.deposit(ng, x, y, z, 2.5)
    expect = -np.ones((ng, ng, ng))
    expect[3, 5, 7] += 2.5
    assert np.array_equal(m[:, :, :ng], expect)
    assert np.all(m[:, :, ng:] == 0)


def test_periodic_wrap_of_deposit(O):
    ng = 8
    m = O.deposit(ng, np.array([7.5]), np.array([7.5]), np.array([7.5]), 8.0)
    d = m[:, :, :ng] + 1
    for i in (7, 0):
        for j in (7, 0):
            for k in (7, 0):
                assert d[i, j, k] == pytest.approx(1.0)
    assert d.sum() == pytest.approx(8.0)


def test_uniform_lattice_gives_zero_everything(O):
    ng = 16
    g = np.arange(ng) + 0.5
    x, y, z = (a.reshape(-1).copy() for a in np.meshgrid(g, g, g, indexing="ij"))
    px, py, pz = (np.zeros_like(x) for _ in range(3))
    cp, ck = O.reference_coefficients()
    delta, phi, f = O.force_step(ng, x, y, z, px, py, pz, 1.0, cp, ck)
    assert np.abs(delta[:, :, :ng]).max() < 1e-14
    assert np.abs(phi[:, :, :ng]).max() < 1e-14
    assert max(np.abs(a).max() for a in f) < 1e-14
    assert max(np.abs(a).max() for a in (px, py, pz)) < 1e-16


@pytest.mark.parametrize("kind", [0, 1])
def test_single_fourier_mode_potential(O, kind):
    """delta = cos(2 pi (a x + b y + c z)/N) -> phi = G(k) N^3 delta."""
    ng = 16
    a, b, c = 1, 2, 3
    i, j, k = np.meshgrid(*(np.arange(ng),) * 3, indexing="ij")
    th = 2 * np.pi * (a * i + b * j + c * k) / ng
    m = O.padded(ng)
    m[:, :, :ng] = np.cos(th)
    cp = 1.7
    O.rfft3d_forward(m)
    O.green(m, cp, kind)
    O.rfft3d_inverse(m)
    w = 2 * np.pi / ng
    if kind == 0:
        lap = -2 * (3 - np.cos(w * a) - np.cos(w * b) - np.cos(w * c))
    else:
        lap = -(w * w) * (a * a + b * b + c * c)
    assert rel(m[:, :, :ng], cp / lap * np.cos(th)) < 1e-13


def test_two_particle_momentum_conservation(O):
    ng = 16
    x, y, z = np.array([3.3, 9.7]), np.array([4.1, 4.6]), np.array([8.2, 12.9])
    px, py, pz = (np.zeros(2) for _ in range(3))
    cp, ck = O.reference_coefficients()
    O.force_step(ng, x, y, z, px, py, pz, 1.0, cp, ck)
    tot = np.array([px.sum(), py.sum(), pz.sum()])
    scale = np.abs(np.concatenate([px, py, pz])).max()
    assert scale > 0
    assert np.abs(tot).max() < 1e-12 * scale


def test_split_join_round_trip(O):
    rng = np.random.default_rng(5)
    ng = 64
    x, y, z = (rng.uniform(0, ng, 1000) for _ in range(3))
    cell, off = O.split_positions(ng, x, y, z)
    xx = O.join_positions(ng, cell, off)
    for a, b in zip((x, y, z), xx):
        assert np.abs(a - b).max() < 2 ** -24


def test_zeldovich_oracle_properties(O):
    ng, nrow = 32, 16
    pos, vel = O.zeldovich_ic(ng, nrow, -2.0, 0.3, seed=7)
    d = np.stack(vel)
    assert np.sqrt(np.mean(np.sum(d * d, axis=0))) == pytest.approx(0.3, rel=1e-12)
    assert all(((p >= 0) & (p < ng)).all() for p in pos)
    w = O.white_noise(7, 1 << 16)
    assert abs(w.mean()) < 0.02 and abs(w.std() - 1) < 0.02
