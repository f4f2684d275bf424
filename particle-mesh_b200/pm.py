"""Python host side of the B200 particle-mesh step, over the C ABI.

``Plan`` wraps one ``pm_plan`` (mesh size, precision, Green's function,
gradient order, CUDA stream) and exposes every stage as a method on torch
CUDA tensors.  Below it, ``deposit_particles``, ``FFT``,
``centered_derivatives`` and ``update_particles`` keep the names and argument
meaning of the reference's CPU functions (include/utils/utils.h:3-10,
include/fft/fftw/fft.h:10-48) so a caller of the reference can switch over
stage by stage.  Tensors must live on the CUDA device of the plan; torch is
used only for device memory and streams.

Errors: the reference has no error reporting (void functions, MPI aborts).
Here every bad argument raises ``PMError`` before any work is enqueued, and
out-of-range positions are reported by ``Plan.check()``.
"""
from __future__ import annotations

import ctypes
import math

import torch

from . import _lib as L
from ._lib import PMError, check

# include/utils/utils_inline.h:13-17
OMEGA_0, OMEGA_M, OMEGA_L = 1.0, 0.3, 0.7
OMEGA_K = 1.0 - OMEGA_M - OMEGA_L
DA, START_A = 0.001, 0.9

_PREC = {"fp64": L.PM_FP64, "fp32": L.PM_FP32}
_GREEN = {"discrete": L.PM_GREEN_DISCRETE, "spectral": L.PM_GREEN_SPECTRAL}


def function_a(a: float) -> float:
    """include/utils/utils_inline.h:51-53."""
    return 1.0 / math.sqrt(OMEGA_M / a + OMEGA_K + OMEGA_L * a * a)


def reference_coefficients(a: float = START_A):
    """(c_poisson, c_kick) of the reference step at scale factor a
    (src/fft/fftw/fft.cpp:55,79 and src/utils/utils.cpp:142)."""
    return 3.0 * OMEGA_0 / (2.0 * a), function_a(a) * DA


def unit_box_coefficients(dt: float, g_m_total: float = 1.0):
    """(c_poisson, c_kick) for a periodic unit box with G M_total = g_m_total,
    positions and velocities in cell units: L Phi = 4 pi G M delta and
    v += -grad Phi dt."""
    return 4.0 * math.pi * g_m_total, dt


def _vp(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _need(t, dtype, numel=None, shape=None, name="tensor"):
    if not isinstance(t, torch.Tensor):
        raise PMError(L.PM_ERR_ARG, f"{name} must be a torch tensor")
    if not t.is_cuda:
        raise PMError(L.PM_ERR_ARG, f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise PMError(L.PM_ERR_ARG, f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise PMError(L.PM_ERR_ARG, f"{name} must be contiguous")
    if numel is not None and t.numel() != numel:
        raise PMError(L.PM_ERR_ARG, f"{name} must have {numel} elements, got {t.numel()}")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise PMError(L.PM_ERR_ARG, f"{name} must have shape {tuple(shape)}, got {tuple(t.shape)}")
    return t


class Plan:
    """One periodic ng^3 box: tables, error word, workspace and a stream."""

    def __init__(self, ng: int, precision: str = "fp64", green: str = "discrete", grad_order: int = 2,
                 stream: torch.cuda.Stream | None = None, device=None):
        self.lib = L.load()
        if precision not in _PREC or green not in _GREEN:
            raise PMError(L.PM_ERR_ARG, f"bad precision {precision!r} or green {green!r}")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.ng, self.precision, self.green_kind, self.grad_order = ng, precision, green, grad_order
        self.dtype = torch.float64 if precision == "fp64" else torch.float32
        with torch.cuda.device(self.device):
            self.stream = stream if stream is not None else torch.cuda.current_stream(self.device)
            h = ctypes.c_void_p()
            check(self.lib.pm_plan_create(ng, _PREC[precision], _GREEN[green], grad_order,
                                          ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self._h = h

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.pm_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def check(self):
        """Raises PMError(PM_ERR_RANGE) if a kernel met a bad position."""
        check(self.lib.pm_plan_check(self._h))

    def device_bytes(self) -> int:
        b = ctypes.c_size_t()
        check(self.lib.pm_plan_device_bytes(self._h, ctypes.byref(b)))
        return b.value

    def set_fft_shape(self, tile_cols: int = 0, radix1: int = 0):
        """Column-tile width and first radix of the strided FFT passes (0: default)."""
        check(self.lib.pm_plan_set_fft_shape(self._h, int(tile_cols), int(radix1)))

    def set_gather(self, mode: str = "cached"):
        """Gather of step_split: "cached" (per particle through L1, the
        default) or "tiled" (bin order, shared-memory tiles; independent of
        the particle order)."""
        modes = {"cached": L.PM_GATHER_CACHED, "tiled": L.PM_GATHER_TILED}
        if mode not in modes:
            raise PMError(L.PM_ERR_ARG, f"unknown gather mode {mode!r}")
        check(self.lib.pm_plan_set_gather(self._h, modes[mode]))

    def set_timing(self, on: bool = True):
        check(self.lib.pm_plan_set_timing(self._h, 1 if on else 0))

    def read_timing(self, reset: bool = True) -> dict:
        """{stage: (milliseconds, launches)} since the last reset."""
        ms = (ctypes.c_double * L.STAGE_COUNT)()
        n = (ctypes.c_int64 * L.STAGE_COUNT)()
        check(self.lib.pm_plan_read_timing(self._h, ms, n, 1 if reset else 0))
        return {self.lib.pm_stage_name(i).decode(): (ms[i], n[i]) for i in range(L.STAGE_COUNT) if n[i]}

    def new_mesh(self) -> torch.Tensor:
        return torch.zeros((self.ng, self.ng, self.ng + 2), dtype=self.dtype, device=self.device)

    def workspace_mesh(self) -> torch.Tensor:
        """The plan's own mesh as a tensor view (no copy)."""
        p = ctypes.c_void_p()
        check(self.lib.pm_plan_mesh(self._h, ctypes.byref(p)))
        n = self.ng
        esz = 8 if self.dtype == torch.float64 else 4
        return _wrap_device_ptr(p.value, (n, n, n + 2), self.dtype, self.device, n * n * (n + 2) * esz)

    def _mesh(self, m, name="mesh"):
        n = self.ng
        return _need(m, self.dtype, shape=(n, n, n + 2), name=name)

    # ------------------------------------------------------------ FP64 stages
    def deposit(self, x, y, z, mass: float, mesh=None):
        mesh = self.new_mesh() if mesh is None else self._mesh(mesh)
        np_ = x.numel()
        for t, nm in ((x, "x"), (y, "y"), (z, "z")):
            _need(t, torch.float64, np_, name=nm)
        check(self.lib.pm_deposit_f64(self._h, _vp(x), _vp(y), _vp(z), np_, float(mass), _vp(mesh)))
        return mesh

    def fft_r2c(self, mesh):
        fn = self.lib.pm_fft_r2c_f64 if self.precision == "fp64" else self.lib.pm_fft_r2c_f32
        check(fn(self._h, _vp(self._mesh(mesh))))
        return mesh

    def fft_c2r(self, mesh):
        fn = self.lib.pm_fft_c2r_f64 if self.precision == "fp64" else self.lib.pm_fft_c2r_f32
        check(fn(self._h, _vp(self._mesh(mesh))))
        return mesh

    def green(self, mesh, c_poisson: float):
        fn = self.lib.pm_green_f64 if self.precision == "fp64" else self.lib.pm_green_f32
        check(fn(self._h, _vp(self._mesh(mesh)), float(c_poisson)))
        return mesh

    def poisson(self, mesh, c_poisson: float):
        fn = self.lib.pm_poisson_f64 if self.precision == "fp64" else self.lib.pm_poisson_f32
        check(fn(self._h, _vp(self._mesh(mesh)), float(c_poisson)))
        return mesh

    def gradient(self, phi, out=None):
        n = self.ng
        if out is None:
            out = [torch.empty((n, n, n), dtype=torch.float64, device=self.device) for _ in range(3)]
        for t, nm in zip(out, ("fx", "fy", "fz")):
            _need(t, torch.float64, shape=(n, n, n), name=nm)
        check(self.lib.pm_gradient_f64(self._h, _vp(self._mesh(phi, "phi")), *(_vp(t) for t in out)))
        return out

    def interp_kick(self, x, y, z, forces, px, py, pz, c_kick: float):
        np_ = x.numel()
        n = self.ng
        for t, nm in ((x, "x"), (y, "y"), (z, "z"), (px, "px"), (py, "py"), (pz, "pz")):
            _need(t, torch.float64, np_, name=nm)
        for t, nm in zip(forces, ("fx", "fy", "fz")):
            _need(t, torch.float64, shape=(n, n, n), name=nm)
        check(self.lib.pm_interp_kick_f64(self._h, _vp(x), _vp(y), _vp(z), *(_vp(t) for t in forces),
                                          _vp(px), _vp(py), _vp(pz), np_, float(c_kick)))

    def drift(self, x, y, z, px, py, pz, dt: float):
        np_ = x.numel()
        for t, nm in ((x, "x"), (y, "y"), (z, "z"), (px, "px"), (py, "py"), (pz, "pz")):
            _need(t, torch.float64, np_, name=nm)
        check(self.lib.pm_drift_f64(self._h, _vp(x), _vp(y), _vp(z), _vp(px), _vp(py), _vp(pz), np_, float(dt)))

    def step(self, x, y, z, px, py, pz, mass: float, c_poisson: float, c_kick: float, dt: float = 0.0):
        np_ = x.numel()
        for t, nm in ((x, "x"), (y, "y"), (z, "z"), (px, "px"), (py, "py"), (pz, "pz")):
            _need(t, torch.float64, np_, name=nm)
        check(self.lib.pm_step_f64(self._h, _vp(x), _vp(y), _vp(z), _vp(px), _vp(py), _vp(pz), np_,
                                   float(mass), float(c_poisson), float(c_kick), float(dt)))

    # ----------------------------------------------------------- adjoints
    def adjoint_deposit(self, x, y, z, mass: float, dbar, xbar):
        np_ = x.numel()
        for t, nm in ((x, "x"), (y, "y"), (z, "z")):
            _need(t, torch.float64, np_, name=nm)
        for t, nm in zip(xbar, ("xbar", "ybar", "zbar")):
            _need(t, torch.float64, np_, name=nm)
        check(self.lib.pm_adjoint_deposit_f64(self._h, _vp(x), _vp(y), _vp(z), np_, float(mass),
                                              _vp(self._mesh(dbar, "dbar")), *(_vp(t) for t in xbar)))

    def adjoint_force(self, x, y, z, mass: float, c_poisson: float, u, scale: float, xbar):
        np_ = x.numel()
        for t, nm in ((x, "x"), (y, "y"), (z, "z")):
            _need(t, torch.float64, np_, name=nm)
        for t in (*u, *xbar):
            _need(t, torch.float64, np_, name="adjoint array")
        check(self.lib.pm_adjoint_force_f64(self._h, _vp(x), _vp(y), _vp(z), np_, float(mass), float(c_poisson),
                                            *(_vp(t) for t in u), float(scale), *(_vp(t) for t in xbar)))

    def step_adjoint(self, x, y, z, mass: float, c_poisson: float, c_kick: float, dt: float, xbar, vbar):
        np_ = x.numel()
        for t, nm in ((x, "x"), (y, "y"), (z, "z")):
            _need(t, torch.float64, np_, name=nm)
        for t in (*xbar, *vbar):
            _need(t, torch.float64, np_, name="adjoint array")
        check(self.lib.pm_step_adjoint_f64(self._h, _vp(x), _vp(y), _vp(z), np_, float(mass), float(c_poisson),
                                           float(c_kick), float(dt), *(_vp(t) for t in xbar),
                                           *(_vp(t) for t in vbar)))

    # ------------------------------------------------- FP32 split positions
    def split(self, x, y, z):
        np_ = x.numel()
        for t, nm in ((x, "x"), (y, "y"), (z, "z")):
            _need(t, torch.float64, np_, name=nm)
        cell = torch.empty(np_, dtype=torch.int32, device=self.device)
        off = [torch.empty(np_, dtype=torch.float32, device=self.device) for _ in range(3)]
        check(self.lib.pm_split_positions(self._h, _vp(x), _vp(y), _vp(z), np_, _vp(cell), *(_vp(t) for t in off)))
        return cell, off

    def join(self, cell, off):
        np_ = cell.numel()
        _need(cell, torch.int32, np_, name="cell")
        for t, nm in zip(off, ("ox", "oy", "oz")):
            _need(t, torch.float32, np_, name=nm)
        out = [torch.empty(np_, dtype=torch.float64, device=self.device) for _ in range(3)]
        check(self.lib.pm_join_positions(self._h, _vp(cell), *(_vp(t) for t in off), np_, *(_vp(t) for t in out)))
        return out

    def _split_args(self, cell, off, vel=None):
        np_ = cell.numel()
        _need(cell, torch.int32, np_, name="cell")
        for t, nm in zip(off, ("ox", "oy", "oz")):
            _need(t, torch.float32, np_, name=nm)
        if vel is not None:
            for t, nm in zip(vel, ("vx", "vy", "vz")):
                _need(t, torch.float32, np_, name=nm)
        return np_

    def deposit_split(self, cell, off, mass: float, mesh=None):
        mesh = self.new_mesh() if mesh is None else self._mesh(mesh)
        np_ = self._split_args(cell, off)
        check(self.lib.pm_deposit_f32(self._h, _vp(cell), *(_vp(t) for t in off), np_, float(mass), _vp(mesh)))
        return mesh

    def sort_split(self, cell, off, vel):
        """Reorders the particle arrays in place into tile Z-order."""
        np_ = self._split_args(cell, off, vel)
        check(self.lib.pm_sort_f32(self._h, _vp(cell), *(_vp(t) for t in off), *(_vp(t) for t in vel), np_))

    def interp_split(self, phi, cell, off):
        np_ = self._split_args(cell, off)
        out = [torch.empty(np_, dtype=torch.float32, device=self.device) for _ in range(3)]
        check(self.lib.pm_interp_f32(self._h, _vp(self._mesh(phi, "phi")), _vp(cell), *(_vp(t) for t in off), np_,
                                     *(_vp(t) for t in out)))
        return out

    def kick_drift_split(self, phi, cell, off, vel, c_kick: float, dt: float):
        np_ = self._split_args(cell, off, vel)
        check(self.lib.pm_kick_drift_f32(self._h, _vp(self._mesh(phi, "phi")), _vp(cell), *(_vp(t) for t in off),
                                         *(_vp(t) for t in vel), np_, float(c_kick), float(dt)))

    def potential_split(self, cell, off, mass: float, c_poisson: float) -> torch.Tensor:
        """The first part of step_split: the particles' potential in the
        workspace mesh (returned); kick_drift_split on it completes the step."""
        np_ = self._split_args(cell, off)
        check(self.lib.pm_potential_f32(self._h, _vp(cell), *(_vp(t) for t in off), np_, float(mass),
                                        float(c_poisson)))
        return self.workspace_mesh()

    def step_split(self, cell, off, vel, mass: float, c_poisson: float, c_kick: float, dt: float):
        np_ = self._split_args(cell, off, vel)
        check(self.lib.pm_step_f32(self._h, _vp(cell), *(_vp(t) for t in off), *(_vp(t) for t in vel), np_,
                                   float(mass), float(c_poisson), float(c_kick), float(dt)))

    # ------------------------------------------------------ FP64 reductions
    def conserved(self, mesh=None, vel=None, mass: float = 1.0) -> dict:
        """Total mass sum(mesh + 1) and momentum mass * sum(v), summed in FP64
        on the device (either input may be None)."""
        out = torch.zeros(4, dtype=torch.float64, device=self.device)
        np_ = 0
        if mesh is not None:
            self._mesh(mesh)
        if vel is not None:
            np_ = vel[0].numel()
            for t, nm in zip(vel, ("vx", "vy", "vz")):
                _need(t, self.dtype, np_, name=nm)
        fn = self.lib.pm_reduce_f64 if self.precision == "fp64" else self.lib.pm_reduce_f32
        check(fn(self._h, _vp(mesh), *(_vp(t) for t in (vel or (None, None, None))), np_, float(mass), _vp(out)))
        o = out.tolist()
        return {"mass": o[0], "momentum": o[1:]}

    # ------------------------------------------- FP32 split-position adjoints
    def _adj_arrays(self, arrays, np_):
        for t in arrays:
            _need(t, torch.float32, np_, name="adjoint array")

    def adjoint_deposit_split(self, cell, off, mass: float, dbar, xbar):
        """xbar += (d delta / d x)^T dbar at the split positions (FP32)."""
        np_ = self._split_args(cell, off)
        self._adj_arrays(xbar, np_)
        check(self.lib.pm_adjoint_deposit_f32(self._h, _vp(cell), *(_vp(t) for t in off), np_, float(mass),
                                              _vp(self._mesh(dbar, "dbar")), *(_vp(t) for t in xbar)))

    def adjoint_force_split(self, cell, off, mass: float, c_poisson: float, u, scale: float, xbar):
        """xbar += scale (dF/dx)^T u, F the FP32 step's forces at the split positions."""
        np_ = self._split_args(cell, off)
        self._adj_arrays((*u, *xbar), np_)
        check(self.lib.pm_adjoint_force_f32(self._h, _vp(cell), *(_vp(t) for t in off), np_, float(mass),
                                            float(c_poisson), *(_vp(t) for t in u), float(scale),
                                            *(_vp(t) for t in xbar)))

    def step_adjoint_split(self, cell, off, mass: float, c_poisson: float, c_kick: float, dt: float, xbar, vbar):
        """The adjoint of one step_split started from (cell, off): (xbar, vbar) in/out."""
        np_ = self._split_args(cell, off)
        self._adj_arrays((*xbar, *vbar), np_)
        check(self.lib.pm_step_adjoint_f32(self._h, _vp(cell), *(_vp(t) for t in off), np_, float(mass),
                                           float(c_poisson), float(c_kick), float(dt), *(_vp(t) for t in xbar),
                                           *(_vp(t) for t in vbar)))


def _wrap_device_ptr(ptr: int, shape, dtype, device, nbytes: int) -> torch.Tensor:
    """A tensor view of device memory owned by a plan (valid while it lives)."""
    class _Arr:
        __cuda_array_interface__ = {
            "shape": tuple(shape), "typestr": "<f8" if dtype == torch.float64 else "<f4",
            "data": (ptr, False), "version": 3, "strides": None,
        }
    return torch.as_tensor(_Arr(), device=device)


def zeldovich_ic(ng: int, nrow: int, n_s: float, rms_cells: float, seed: int, vel_factor: float = 1.0,
                 device=None, stream: torch.cuda.Stream | None = None):
    """Zel'dovich particles (positions, velocities; FP64 device tensors)."""
    lib = L.load()
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    n3 = nrow ** 3
    pos = [torch.empty(n3, dtype=torch.float64, device=dev) for _ in range(3)]
    vel = [torch.empty(n3, dtype=torch.float64, device=dev) for _ in range(3)]
    with torch.cuda.device(dev):
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        check(lib.pm_ic_zeldovich(ng, nrow, float(n_s), float(rms_cells), int(seed) & (2 ** 64 - 1),
                                  float(vel_factor), *(_vp(t) for t in pos), *(_vp(t) for t in vel),
                                  ctypes.c_void_p(s.cuda_stream)))
    return pos, vel


class Ensemble:
    """Independent boxes of mixed mesh sizes advanced together (FP32 split).

    Particles of all boxes live in one set of split arrays, box b owning
    np[b] consecutive entries."""

    def __init__(self, ng, np, mass, green: str = "spectral", grad_order: int = 4, autotune: bool = True,
                 tune_cache: str | None = None, stream: torch.cuda.Stream | None = None):
        self.lib = L.load()
        n = len(ng)
        self.ng, self.np = list(ng), list(np)
        a_ng = (ctypes.c_int * n)(*ng)
        a_np = (ctypes.c_int64 * n)(*np)
        a_m = (ctypes.c_float * n)(*mass)
        # a stream of its own (graphs are not captured on the legacy stream),
        # ordered against the caller's current stream around every call
        self.stream = stream if stream is not None else torch.cuda.Stream()
        h = ctypes.c_void_p()
        check(self.lib.pm_ensemble_create(n, a_ng, a_np, a_m, _GREEN[green], grad_order, 1 if autotune else 0,
                                          tune_cache.encode() if tune_cache else None,
                                          ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.pm_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def info(self) -> dict:
        nc = ctypes.c_int()
        ng = (ctypes.c_int * 64)()
        nb = (ctypes.c_int * 64)()
        tk = (ctypes.c_int * 64)()
        r1 = (ctypes.c_int * 64)()
        by = ctypes.c_size_t()
        nodes = ctypes.c_size_t()
        check(self.lib.pm_ensemble_info(self._h, ctypes.byref(nc), ng, nb, tk, r1, ctypes.byref(by),
                                        ctypes.byref(nodes)))
        return {"classes": [{"ng": ng[i], "boxes": nb[i], "tile_cols": tk[i], "radix1": r1[i]} for i in range(nc.value)],
                "device_bytes": by.value, "graph_nodes": nodes.value}

    def step(self, cell, off, vel, c_poisson: float, c_kick: float, dt: float):
        cur = torch.cuda.current_stream()
        self.stream.wait_stream(cur)
        check(self.lib.pm_ensemble_step_f32(self._h, _vp(cell), *(_vp(t) for t in off), *(_vp(t) for t in vel),
                                            float(c_poisson), float(c_kick), float(dt)))
        cur.wait_stream(self.stream)

    def run(self, cell, off, vel, c_poisson: float, dt: float, steps: int):
        """`steps` KDK steps as one CUDA graph (captured on first use)."""
        cur = torch.cuda.current_stream()
        self.stream.wait_stream(cur)
        check(self.lib.pm_ensemble_run_f32(self._h, _vp(cell), *(_vp(t) for t in off), *(_vp(t) for t in vel),
                                           float(c_poisson), float(dt), int(steps)))
        cur.wait_stream(self.stream)


# ------------------------------------------------ reference-named mirrors
_plans: dict = {}


def _default_plan(ng: int, device) -> Plan:
    key = (ng, str(device))
    if key not in _plans:
        _plans[key] = Plan(ng, "fp64", "discrete", 2, device=device)
    return _plans[key]


def deposit_particles(posx, posy, posz, buf, mass: float, plan: Plan | None = None):
    """CIC deposit of the density contrast into buf [ng][ng][ng+2] (FP64).

    Mirrors deposit_particles (src/utils/utils.cpp:70-102) together with the
    init_buf / reduce_private_to_shared / TransposeSlab / ReorderSlab stages
    that bracket it in the reference loop (src/core/main.cpp:93-106)."""
    plan = plan or _default_plan(buf.shape[0], buf.device)
    return plan.deposit(posx, posy, posz, mass, buf)


class FFT:
    """In-place 3D R2C / C2R on a [ng][ng][ng+2] FP64 buffer with the
    reference's Green's function; mirrors class FFT
    (include/fft/fftw/fft.h:10-48, src/fft/fftw/fft.cpp)."""

    def __init__(self, n: int, buf: torch.Tensor, plan: Plan | None = None):
        self.n = n
        self.buf = buf
        self.plan = plan or _default_plan(n, buf.device)

    def forward(self):  # src/fft/fftw/fft.cpp:96
        self.plan.fft_r2c(self.buf)

    def backward(self):  # src/fft/fftw/fft.cpp:97
        self.plan.fft_c2r(self.buf)

    def apply_green(self, a: float):  # src/fft/fftw/fft.cpp:75-82
        self.plan.green(self.buf, 3.0 * OMEGA_0 / (2.0 * a))

    # the single-box slab is the whole mesh
    def local_n0(self):
        return self.n

    def local_0_start(self):
        return 0

    def local_alloc(self):
        return self.n * self.n * (self.n // 2 + 1)


def centered_derivatives(inp, d_dx, d_dy, d_dz, plan: Plan | None = None):
    """-grad(phi) by 2-point centred differences (src/utils/utils.cpp:115-137)
    with the ghost exchange of the reference replaced by periodic wraps."""
    plan = plan or _default_plan(inp.shape[0], inp.device)
    return plan.gradient(inp, [d_dx, d_dy, d_dz])


def update_particles(posx, posy, posz, d_dx, d_dy, d_dz, px, py, pz, a: float, plan: Plan | None = None):
    """p += g * function_a(a) * Da with g the CIC-interpolated force
    (src/utils/utils.cpp:141-170)."""
    plan = plan or _default_plan(d_dx.shape[0], d_dx.device)
    plan.interp_kick(posx, posy, posz, (d_dx, d_dy, d_dz), px, py, pz, function_a(a) * DA)


# ----------------------------------------------- cosmological time stepping
def cosmo_schedule(a0: float = START_A, da: float = DA, nsteps: int = 1):
    """Leapfrog KDK in the scale factor, the integration the reference sketches
    in update_particles (src/utils/utils.cpp:141-143): force evaluation
    s = 0..nsteps at a_s = a0 + s da with Poisson prefactor 3 Omega_0 / (2 a_s)
    (src/fft/fftw/fft.cpp:55) and kick function_a(a_s) da (halved at the two
    ends, the inner half kicks merged); after evaluation s < nsteps a drift of
    a^-2 function_a(a) da at a = a0 + (s + 1/2) da.  One (a, c_poisson,
    c_kick, dt) tuple per Plan.step / Plan.step_split call."""
    out = []
    for s in range(nsteps + 1):
        a = a0 + s * da
        ah = a0 + (s + 0.5) * da
        w = 0.5 if s in (0, nsteps) else 1.0
        out.append((a, 3.0 * OMEGA_0 / (2.0 * a), w * function_a(a) * da,
                    function_a(ah) * da / (ah * ah) if s < nsteps else 0.0))
    return out


def cosmo_run(plan: Plan, pos, mom, mass: float, a0: float = START_A, da: float = DA, nsteps: int = 1):
    """Advances FP64 positions / momenta (or, on an FP32 plan, split positions
    (cell, off) and FP32 velocities) through cosmo_schedule; returns the final
    scale factor."""
    for _, cp, ck, dt in cosmo_schedule(a0, da, nsteps):
        if plan.precision == "fp64":
            plan.step(*pos, *mom, mass, cp, ck, dt)
        else:
            plan.step_split(pos[0], pos[1], mom, mass, cp, ck, dt)
    return a0 + nsteps * da


# -------------------------------------------------------------- snapshots
# Little-endian file: a 72-byte header, then x, y, z (cell units), vx, vy, vz
# as float64 arrays of np values.  The reference writes no output; this is
# the format of the C++ mirror's pm::write_snapshot as well.
_SNAP_MAGIC = b"PMSNAP1\0"
_SNAP_HEAD = "<8sIIqqddddd"


def write_snapshot(path: str, ng: int, a: float, mass: float, pos, vel):
    """Writes positions and velocities (any device, any float dtype)."""
    import struct
    np_ = pos[0].numel()
    with open(path, "wb") as f:
        f.write(struct.pack(_SNAP_HEAD, _SNAP_MAGIC, 1, 0, ng, np_, float(a), float(mass), OMEGA_M, OMEGA_L,
                            OMEGA_0))
        for t in (*pos, *vel):
            if t.numel() != np_:
                raise PMError(L.PM_ERR_ARG, "snapshot arrays must all have np values")
            f.write(t.detach().to("cpu", torch.float64).contiguous().numpy().tobytes())


def read_snapshot(path: str) -> dict:
    """{ng, np, a, mass, omega_m, omega_lambda, omega_0, pos: [3], vel: [3]}
    (float64 CPU tensors)."""
    import struct
    size = struct.calcsize(_SNAP_HEAD)
    with open(path, "rb") as f:
        head = f.read(size)
        if len(head) != size:
            raise PMError(L.PM_ERR_ARG, f"{path}: truncated header")
        magic, ver, _flags, ng, np_, a, mass, om, ol, o0 = struct.unpack(_SNAP_HEAD, head)
        if magic != _SNAP_MAGIC or ver != 1:
            raise PMError(L.PM_ERR_ARG, f"{path}: not a version-1 particle-mesh snapshot")
        body = f.read()
    if len(body) != 6 * 8 * np_:
        raise PMError(L.PM_ERR_ARG, f"{path}: expected {6 * 8 * np_} bytes of particle data, got {len(body)}")
    arr = torch.frombuffer(bytearray(body), dtype=torch.float64).view(6, np_)
    return {"ng": ng, "np": np_, "a": a, "mass": mass, "omega_m": om, "omega_lambda": ol, "omega_0": o0,
            "pos": [arr[i].clone() for i in range(3)], "vel": [arr[3 + i].clone() for i in range(3)]}
