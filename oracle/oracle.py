"""CPU oracle for the particle-mesh step.

TEST INFRASTRUCTURE, NOT PRODUCT.  Only tests/, ``__graft_entry__.smoke()`` and
``bench.py``'s cpu_baseline / reference legs may import this module, and only as
the checker or as the timed CPU baseline.  The CUDA path never calls it.

Two CPU implementations live here:

* the restatement (``liboracle.so`` built from ``pm_oracle.c``): this project's
  FP64 C code for every stage of the reference step on one periodic box;
* the reference itself (``_ref/libpmref*.so``): the reference's own
  ``src/utils/utils.cpp`` and ``src/decomp/slab/reorder_slab{,_back}.cpp``
  compiled from their sources by ``oracle/Makefile``.  The reference's FFT
  (FFTW3-MPI or the vendored FFTE Fortran) cannot be built here, so the
  reference pipeline uses ``numpy.fft`` (pocketfft, FP64) as the DFT; the
  reference's Green's table (src/fft/fftw/fft.cpp:50-57) is restated in numpy.

Zel'dovich initial conditions and the split-position helpers are new (the
reference only draws uniform positions, src/utils/utils.cpp:22-36); their
restatement lives here too so the GPU generator can be checked.
"""
from __future__ import annotations

import ctypes
import os
import platform
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_dp = ctypes.POINTER(ctypes.c_double)
_lib = None
_ref = None


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def lib():
    """The restatement library, built with gcc on first use if missing."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
        L = ctypes.CDLL(path)
        i, l, d = ctypes.c_int, ctypes.c_long, ctypes.c_double
        L.orc_deposit.argtypes = [i, l, _dp, _dp, _dp, d, _dp]
        L.orc_fft1d.argtypes = [l, _dp, l, i]
        L.orc_rfft3d_forward.argtypes = [i, _dp]
        L.orc_rfft3d_inverse.argtypes = [i, _dp]
        L.orc_green.argtypes = [i, _dp, d, i]
        L.orc_gradient.argtypes = [i, i, _dp, _dp, _dp, _dp]
        L.orc_interp_kick.argtypes = [i, l, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, d]
        L.orc_drift.argtypes = [i, l, _dp, _dp, _dp, _dp, _dp, _dp, d]
        _lib = L
    return _lib


def _cpu_has_v3() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            flags = next((ln for ln in f if ln.startswith("flags")), "")
        return all(x in flags.split() for x in ("avx2", "fma", "bmi2"))
    except OSError:
        return False


def ref_lib():
    """The reference's own kernels (oracle/_ref), or None if not built.

    Built from the reference sources by oracle/Makefile (target
    ref-if-present: the tree named by PM_REFERENCE_DIR, or the Makefile's
    default) when they are present on this machine; elsewhere only a
    prebuilt copy can be used."""
    global _ref
    if _ref is not None:
        return _ref
    d = os.path.join(HERE, "_ref")
    names = (["libpmref_v3.so"] if _cpu_has_v3() and platform.machine() == "x86_64" else []) + ["libpmref.so"]
    paths = [os.path.join(d, n) for n in names]
    if not any(os.path.exists(p) for p in paths):
        subprocess.run(["make", "-s", "-C", HERE, "ref-if-present"], check=True)
    path = next((p for p in paths if os.path.exists(p)), None)
    if path is None:
        return None
    L = ctypes.CDLL(path)
    i, l, d, sz = ctypes.c_int, ctypes.c_long, ctypes.c_double, ctypes.c_size_t
    ip = ctypes.POINTER(ctypes.c_int)
    L.ref_set_threads.argtypes = [i]
    L.ref_max_threads.restype = i
    L.ref_init_particles.argtypes = [_dp, _dp, _dp, sz, i, i, i, i, i, i, i]
    L.ref_init_buf.argtypes = [_dp, i, i, i, sz, i]
    L.ref_deposit_particles.argtypes = [_dp, _dp, _dp, sz, _dp, sz, i, i, i, i, i, i, d]
    L.ref_reduce_private_to_shared.argtypes = [_dp, sz, i]
    L.ref_centered_derivatives.argtypes = [_dp, _dp, _dp, _dp, i, i, i]
    L.ref_update_particles.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, d, sz, i, i, i, i, i]
    L.ref_function_a.argtypes = [d]
    L.ref_function_a.restype = d
    L.ref_constants.argtypes = [_dp]
    L.ref_reorder_slab_create.argtypes = [i, i, i, l, i, ip, ip, i, ip]
    L.ref_reorder_slab_create.restype = ctypes.c_void_p
    L.ref_reorder_slab_execute.argtypes = [ctypes.c_void_p, _dp, _dp]
    L.ref_reorder_slab_destroy.argtypes = [ctypes.c_void_p]
    L.ref_reorder_slab_back_create.argtypes = [i, i, i, i, ip, l]
    L.ref_reorder_slab_back_create.restype = ctypes.c_void_p
    L.ref_reorder_slab_back_execute.argtypes = [ctypes.c_void_p, _dp, _dp]
    L.ref_reorder_slab_back_destroy.argtypes = [ctypes.c_void_p]
    _ref = L
    return _ref


# ----------------------------------------------------------------- constants
# include/utils/utils_inline.h:13-17
OMEGA_0, OMEGA_M, OMEGA_L = 1.0, 0.3, 0.7
OMEGA_K = 1.0 - OMEGA_M - OMEGA_L
DA, START_A = 0.001, 0.9


def function_a(a: float) -> float:
    """include/utils/utils_inline.h:51-53."""
    return 1.0 / np.sqrt(OMEGA_M / a + OMEGA_K + OMEGA_L * a * a)


def reference_coefficients(a: float = START_A):
    """(c_poisson, c_kick) that reproduce the reference step at scale factor a.

    Green: -3 Omega_0 / (4 N^3 (3 - sum cos)) / a  (src/fft/fftw/fft.cpp:55,79)
         = -c_poisson / (2 N^3 (3 - sum cos)) with c_poisson = 3 Omega_0 / (2a).
    Kick:  p += g * function_a(a) * Da             (src/utils/utils.cpp:142,166)."""
    return 3.0 * OMEGA_0 / (2.0 * a), function_a(a) * DA


# ------------------------------------------------------------- restatement

def padded(ng: int) -> np.ndarray:
    return np.zeros((ng, ng, ng + 2), np.float64)


def spectrum_view(mesh: np.ndarray) -> np.ndarray:
    """Complex [kx][ky][kz] view of a padded real mesh [ng][ng][ng+2]."""
    return mesh.view(np.complex128)


def deposit(ng, x, y, z, mass):
    m = padded(ng)
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
    lib().orc_deposit(ng, x.size, _ptr(x), _ptr(y), _ptr(z), float(mass), _ptr(m))
    return m


def rfft3d_forward(mesh):
    lib().orc_rfft3d_forward(mesh.shape[0], _ptr(mesh))
    return mesh


def rfft3d_inverse(mesh):
    lib().orc_rfft3d_inverse(mesh.shape[0], _ptr(mesh))
    return mesh


def green(mesh, c, kind=0):
    lib().orc_green(mesh.shape[0], _ptr(mesh), float(c), int(kind))
    return mesh


def fft1d(a: np.ndarray, sign=-1):
    b = np.ascontiguousarray(a, np.complex128).copy()
    lib().orc_fft1d(b.size, b.view(np.float64).ctypes.data_as(_dp), 1, int(sign))
    return b


def gradient(phi, order=2):
    ng = phi.shape[0]
    f = [np.zeros((ng, ng, ng), np.float64) for _ in range(3)]
    lib().orc_gradient(ng, int(order), _ptr(phi), *(_ptr(a) for a in f))
    return f


def interp_kick(x, y, z, f, px, py, pz, c_kick):
    ng = f[0].shape[0]
    lib().orc_interp_kick(ng, x.size, _ptr(x), _ptr(y), _ptr(z), *(_ptr(a) for a in f),
                          _ptr(px), _ptr(py), _ptr(pz), float(c_kick))


def drift(ng, x, y, z, px, py, pz, dt):
    lib().orc_drift(ng, x.size, _ptr(x), _ptr(y), _ptr(z), _ptr(px), _ptr(py), _ptr(pz), float(dt))


def green_table(ng: int, c: float, kind: int = 0) -> np.ndarray:
    """The Green's factors of orc_green as a [kx][ky][kz] table (numpy)."""
    n = ng
    i = np.arange(n)[:, None, None]
    j = np.arange(n)[None, :, None]
    k = np.arange(n // 2 + 1)[None, None, :]
    w = 2.0 * np.pi / n
    with np.errstate(divide="ignore", invalid="ignore"):
        if kind == 0:
            g = -c / (2.0 * float(n) ** 3 * (3 - np.cos(w * i) - np.cos(w * j) - np.cos(w * k)))
        else:
            mi = np.where(i <= n // 2, i, i - n)
            mj = np.where(j <= n // 2, j, j - n)
            g = -c / (float(n) ** 3 * (w * w) * (mi * mi + mj * mj + k * k))
    g[0, 0, 0] = 0.0
    return g


def potential(ng, x, y, z, mass, c_poisson, green_kind=0, fft="auto"):
    """delta -> phi (padded real mesh).  fft="c" uses the restated FFT,
    "numpy" pocketfft (faster for large meshes); "auto" picks numpy from
    ng >= 128."""
    m = deposit(ng, x, y, z, mass)
    delta = m.copy()
    if fft == "c" or (fft == "auto" and ng < 128):
        rfft3d_forward(m)
        green(m, c_poisson, green_kind)
        rfft3d_inverse(m)
    else:
        spec = np.fft.rfftn(m[:, :, :ng]) * green_table(ng, c_poisson, green_kind)
        m[:, :, :ng] = np.fft.irfftn(spec, s=(ng, ng, ng), axes=(0, 1, 2)) * float(ng) ** 3
        m[:, :, ng:] = 0.0
    return delta, m


def force_step(ng, x, y, z, px, py, pz, mass, c_poisson, c_kick, green_kind=0, grad_order=2, fft="auto"):
    """One reference step (deposit, Poisson, gradient, interpolate, kick) in
    place on px, py, pz.  Returns (delta, phi, forces)."""
    delta, phi = potential(ng, x, y, z, mass, c_poisson, green_kind, fft)
    f = gradient(phi, grad_order)
    interp_kick(x, y, z, f, px, py, pz, c_kick)
    return delta, phi, f


def kdk(ng, x, y, z, vx, vy, vz, mass, c_poisson, dt, steps, green_kind=1, grad_order=4):
    """Leapfrog kick-drift-kick: steps+1 force evaluations, with the inner
    half kicks merged (K(dt/2) D F K(dt) D ... F K(dt/2)).  New: the reference
    has no drift (src/core/main.cpp:90-139)."""
    for s in range(steps + 1):
        ck = 0.5 * dt if s in (0, steps) else dt
        force_step(ng, x, y, z, vx, vy, vz, mass, c_poisson, ck, green_kind, grad_order)
        if s < steps:
            drift(ng, x, y, z, vx, vy, vz, dt)


def function_a(a: float) -> float:
    """include/utils/utils_inline.h:51-53 with Omega_m = 0.3, Omega_lambda = 0.7."""
    return 1.0 / np.sqrt(0.3 / a + 0.0 + 0.7 * a * a)


def cosmo_kdk(ng, x, y, z, px, py, pz, mass, a0, da, steps, green_kind=0, grad_order=2):
    """Leapfrog KDK in the scale factor (new: src/utils/utils.cpp:141-143
    sketches it): force s at a_s = a0 + s da with c_poisson = 3 / (2 a_s) and
    kick function_a(a_s) da (halved at both ends), drift a^-2 function_a(a) da
    at a = a0 + (s + 1/2) da."""
    for s in range(steps + 1):
        a = a0 + s * da
        w = 0.5 if s in (0, steps) else 1.0
        force_step(ng, x, y, z, px, py, pz, mass, 3.0 / (2.0 * a), w * function_a(a) * da, green_kind, grad_order)
        if s < steps:
            ah = a0 + (s + 0.5) * da
            drift(ng, x, y, z, px, py, pz, function_a(ah) * da / (ah * ah))


# ------------------------------------------------ the reference, single box

def green_table_reference(ng: int, c_poisson: float) -> np.ndarray:
    """Green's table of src/fft/fftw/fft.cpp:50-57 in [kx][ky][kz] order, times
    the reference's 1/a folded into c_poisson (fft.cpp:75-82)."""
    n = ng
    i = np.arange(n)[:, None, None]
    j = np.arange(n)[None, :, None]
    k = np.arange(n // 2 + 1)[None, None, :]
    pi_n = 2.0 * np.pi / n
    with np.errstate(divide="ignore"):
        g = -c_poisson / (2.0 * (float(n) ** 3) * (3 - np.cos(pi_n * i) - np.cos(pi_n * j) - np.cos(pi_n * k)))
    g[0, 0, 0] = 0.0
    return g


class ReferenceStepper:
    """The reference step at P = 1 through the reference's own compiled code,
    with its setup done once as in src/core/main.cpp:42-69 (buffers, FFT /
    Green's table, ReorderSlab / ReorderSlabBack plans).

    Stages of step() (src/core/main.cpp:90-139):
      init_buf + deposit_particles + reduce_private_to_shared   (reference code)
      TransposeSlab: at P = 1 the exchange is the identity on the (ng+1)^3
        cube; ReorderSlab folds the x = ng ghost plane as its own chunk
        (the single-rank form of transpose_slab.cpp:23-27)      (reference code)
      FFT forward / Green / FFT backward: numpy.fft (or a drop-in such as
        scipy.fft) stands in for FFTW; Green's table of fft.cpp:50-57
      ReorderSlabBack (y, z ghosts)                             (reference code)
      TransposeSlabBack: x ghosts -1/+2 as periodic planes (the single-rank
        form of transpose_slab_back.cpp:22-44)
      centered_derivatives + update_particles                   (reference code)
    The per-stage wall times accumulate in .timers (seconds), the reference's
    own 9 buckets (main.cpp:88-143)."""

    BUCKETS = ("cic", "alltoallv", "reorder", "fft", "green", "ifft", "reorder_back", "alltoallv_back", "update")

    def __init__(self, ng, a=START_A, threads=None, rfftn=None, irfftn=None):
        R = ref_lib()
        if R is None:
            raise RuntimeError("oracle/_ref is not built")
        self.R, self.ng, self.a = R, ng, a
        self.T = int(threads or R.ref_max_threads())
        self.rfftn = rfftn or np.fft.rfftn
        self.irfftn = irfftn or (lambda s_, **k: np.fft.irfftn(s_, **k))
        n = ng
        self.nx = n + 1
        self.ncell = self.nx ** 3
        self.buf = np.empty(self.T * self.ncell, np.float64)
        self.stride = n + 2
        rc = (ctypes.c_int * 2)(n * self.nx * self.nx, self.nx * self.nx)
        rd = (ctypes.c_int * 2)(0, n * self.nx * self.nx)
        dims = (ctypes.c_int * 3)(2, 1, 1)
        self.h = R.ref_reorder_slab_create(n, self.nx, self.nx, n, self.stride, rc, rd, 2, dims)
        dims1 = (ctypes.c_int * 3)(1, 1, 1)
        self.hb = R.ref_reorder_slab_back_create(n, n, n, self.stride, dims1, n)
        self.green = green_table_reference(n, 3.0 * OMEGA_0 / (2.0 * a))
        self.slab = np.zeros((n, n, self.stride), np.float64)
        self.phi = np.zeros((n, n, self.stride), np.float64)
        self.yz = np.zeros((n, n + 3, n + 3), np.float64)
        self.ghost_index = (np.arange(n + 3) - 1) % n
        self.d = [np.zeros(self.ncell, np.float64) for _ in range(3)]
        self.timers = {b: 0.0 for b in self.BUCKETS}

    def close(self):
        if self.h:
            self.R.ref_reorder_slab_destroy(self.h)
            self.R.ref_reorder_slab_back_destroy(self.hb)
            self.h = self.hb = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def step(self, x, y, z, px, py, pz, mass):
        import time
        R, n, T = self.R, self.ng, self.T
        R.ref_set_threads(T)
        clock = time.perf_counter
        t = [clock()]

        def mark(name):
            t.append(clock())
            self.timers[name] += t[-1] - t[-2]

        nx = self.nx
        R.ref_init_buf(_ptr(self.buf), nx, nx, nx, self.ncell, T)
        R.ref_deposit_particles(_ptr(x), _ptr(y), _ptr(z), x.size, _ptr(self.buf), self.ncell, nx, nx, nx,
                                0, 0, 0, float(mass))
        R.ref_reduce_private_to_shared(_ptr(self.buf), self.ncell, T)
        mark("cic")
        mark("alltoallv")  # identity at P = 1: the recv buffer is the cube itself
        R.ref_reorder_slab_execute(self.h, _ptr(self.buf), _ptr(self.slab))
        mark("reorder")
        delta = self.slab.copy() if self.keep else None
        spec = self.rfftn(self.slab[:, :, :n])
        mark("fft")
        spec *= self.green
        mark("green")
        self.phi[:, :, :n] = self.irfftn(spec, s=(n, n, n), axes=(0, 1, 2))
        self.phi[:, :, :n] *= float(n) ** 3
        mark("ifft")
        R.ref_reorder_slab_back_execute(self.hb, _ptr(self.phi), _ptr(self.yz))
        mark("reorder_back")
        ghost = np.ascontiguousarray(self.yz[self.ghost_index])
        mark("alltoallv_back")
        R.ref_centered_derivatives(_ptr(ghost), *(_ptr(a) for a in self.d), n + 3, n + 3, n + 3)
        R.ref_update_particles(_ptr(x), _ptr(y), _ptr(z), *(_ptr(a) for a in self.d), _ptr(px), _ptr(py),
                               _ptr(pz), float(self.a), x.size, nx, nx, 0, 0, 0)
        mark("update")
        if not self.keep:
            return None
        return {"delta": delta, "phi": self.phi.copy(), "forces": [a.reshape(nx, nx, nx).copy() for a in self.d]}

    keep = True


def reference_force_step(ng, x, y, z, px, py, pz, mass, a=START_A, threads=None, timers=None):
    """One reference step at P = 1 (see ReferenceStepper); returns dict with
    delta (slab), phi (slab), forces ((ng+1)^3 each)."""
    st = ReferenceStepper(ng, a, threads)
    try:
        r = st.step(x, y, z, px, py, pz, mass)
        if timers is not None:
            for k, v in st.timers.items():
                timers[k] = timers.get(k, 0.0) + v
        return r
    finally:
        st.close()


def reference_init_particles(ng: int, nrow: int, rank: int = 0):
    """Uniform positions of src/utils/utils.cpp:22-36 at P = 1 (seeds 0, 1, 2)."""
    R = ref_lib()
    np_ = nrow ** 3
    x, y, z = (np.empty(np_, np.float64) for _ in range(3))
    R.ref_init_particles(_ptr(x), _ptr(y), _ptr(z), np_, 0, 0, 0, ng, ng, ng, rank)
    return x, y, z


# ------------------------------------------------- Zel'dovich initial state

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(z: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser (Steele, Lea, Flood 2014), vectorised on uint64."""
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def white_noise(seed: int, n: int) -> np.ndarray:
    """N(0,1) deviates, one per lattice site, by Box-Muller on two counter
    hashes: key = splitmix64(seed); u1 = (hash(key ^ 2i) >> 11 + 1) 2^-53,
    u2 = (hash(key ^ (2i+1)) >> 11) 2^-53, g = sqrt(-2 ln u1) cos(2 pi u2)."""
    key = splitmix64(np.array([seed], np.uint64))[0]
    idx = np.arange(n, dtype=np.uint64)
    h1 = splitmix64(key ^ (idx * np.uint64(2)))
    h2 = splitmix64(key ^ (idx * np.uint64(2) + np.uint64(1)))
    u1 = ((h1 >> np.uint64(11)).astype(np.float64) + 1.0) * 2.0 ** -53
    u2 = (h2 >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def zeldovich_displacement(nrow: int, n_s: float, seed: int) -> np.ndarray:
    """Unnormalised displacement field psi[3][nrow][nrow][nrow] in lattice
    units: psi_hat_a = i k_a / k^2 * W_hat * |k|^(n_s/2), W white noise,
    k_a = 0 on its Nyquist plane, psi_hat(0) = 0."""
    w = white_noise(seed, nrow ** 3).reshape(nrow, nrow, nrow)
    W = np.fft.rfftn(w)
    kf = 2.0 * np.pi * np.fft.fftfreq(nrow)
    kr = 2.0 * np.pi * np.fft.rfftfreq(nrow)
    kx, ky, kz = kf[:, None, None], kf[None, :, None], kr[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = 1.0
    amp = k2 ** (n_s / 4.0)
    amp[0, 0, 0] = 0.0
    D = W * amp / k2
    out = []
    for ka, ax in ((kx, 0), (ky, 1), (kz, 2)):
        ka = np.array(ka, copy=True)
        sl = [slice(None)] * 3
        sl[ax] = nrow // 2
        ka[tuple(sl)] = 0.0
        out.append(np.fft.irfftn(1j * ka * D, s=(nrow, nrow, nrow), axes=(0, 1, 2)))
    return np.stack(out)


def zeldovich_ic(ng: int, nrow: int, n_s: float, rms_cells: float, seed: int, vel_factor: float = 1.0):
    """Particles on the nrow^3 lattice q = (i + 1/2) ng/nrow, displaced by the
    Zel'dovich field scaled so that sqrt(<|psi|^2>) = rms_cells (cell units),
    velocities vel_factor * psi.  Lagrangian order, k fastest."""
    psi = zeldovich_displacement(nrow, n_s, seed)
    sp = ng / nrow
    rms = np.sqrt(np.mean(np.sum(psi * psi, axis=0))) * sp
    s = sp * (rms_cells / rms if rms > 0 else 0.0)
    d = psi.reshape(3, -1) * s
    i = np.arange(nrow)
    q = [(np.broadcast_to(g, (nrow,) * 3).reshape(-1) + 0.5) * sp
         for g in (i[:, None, None], i[None, :, None], i[None, None, :])]
    pos = [np.mod(q[a] + d[a], float(ng)) for a in range(3)]
    pos = [np.where(p >= ng, p - ng, p) for p in pos]
    vel = [vel_factor * d[a] for a in range(3)]
    return pos, vel


# --------------------------------------------------------- split positions

def split_positions(ng: int, x, y, z):
    """(cell index (ix*ng + iy)*ng + iz as uint32, FP32 in-cell offsets).

    New: the reference stores FP64 positions only."""
    f = [np.floor(a) for a in (x, y, z)]
    c = [np.mod(fa.astype(np.int64), ng) for fa in f]
    off = [(a - fa).astype(np.float32) for a, fa in zip((x, y, z), f)]
    cell = ((c[0] * ng + c[1]) * ng + c[2]).astype(np.uint32)
    return cell, off


def join_positions(ng: int, cell, off):
    cell = cell.astype(np.int64)
    ix, iy, iz = cell // (ng * ng), (cell // ng) % ng, cell % ng
    return [i.astype(np.float64) + o.astype(np.float64) for i, o in zip((ix, iy, iz), off)]
