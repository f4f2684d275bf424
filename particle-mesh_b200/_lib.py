"""ctypes binding of the C ABI in include/pm_b200.h (libpm_b200.so).

The library is the CUDA build of this package; there is no CPU fallback.
Loading fails loudly when the library is missing and cannot be built.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpm_b200.so")

PM_OK, PM_ERR_ARG, PM_ERR_SIZE, PM_ERR_CUDA, PM_ERR_NOMEM, PM_ERR_RANGE, PM_ERR_STATE = range(7)
PM_FP64, PM_FP32 = 0, 1
PM_GREEN_DISCRETE, PM_GREEN_SPECTRAL = 0, 1
PM_GATHER_CACHED, PM_GATHER_TILED = 0, 1
PM_IPC_HANDLE_BYTES = 64

_STATUS = {PM_ERR_ARG: "PM_ERR_ARG", PM_ERR_SIZE: "PM_ERR_SIZE", PM_ERR_CUDA: "PM_ERR_CUDA",
           PM_ERR_NOMEM: "PM_ERR_NOMEM", PM_ERR_RANGE: "PM_ERR_RANGE", PM_ERR_STATE: "PM_ERR_STATE"}

# Every function of the ABI with its argument types (p = pointer / handle).
_V, _I, _L, _D, _F, _U64, _SZ = (ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double,
                                 ctypes.c_float, ctypes.c_uint64, ctypes.c_size_t)
SIGNATURES = {
    "pm_plan_create": [_I, _I, _I, _I, _V, ctypes.POINTER(_V)],
    "pm_plan_destroy": [_V],
    "pm_plan_device_bytes": [_V, ctypes.POINTER(_SZ)],
    "pm_plan_check": [_V],
    "pm_plan_mesh": [_V, ctypes.POINTER(_V)],
    "pm_plan_set_timing": [_V, _I],
    "pm_plan_read_timing": [_V, _V, _V, _I],
    "pm_deposit_f64": [_V, _V, _V, _V, _L, _D, _V],
    "pm_fft_r2c_f64": [_V, _V],
    "pm_green_f64": [_V, _V, _D],
    "pm_fft_c2r_f64": [_V, _V],
    "pm_poisson_f64": [_V, _V, _D],
    "pm_gradient_f64": [_V, _V, _V, _V, _V],
    "pm_interp_kick_f64": [_V, _V, _V, _V, _V, _V, _V, _V, _V, _V, _L, _D],
    "pm_drift_f64": [_V, _V, _V, _V, _V, _V, _V, _L, _D],
    "pm_step_f64": [_V, _V, _V, _V, _V, _V, _V, _L, _D, _D, _D, _D],
    "pm_adjoint_deposit_f64": [_V, _V, _V, _V, _L, _D, _V, _V, _V, _V],
    "pm_adjoint_force_f64": [_V, _V, _V, _V, _L, _D, _D, _V, _V, _V, _D, _V, _V, _V],
    "pm_step_adjoint_f64": [_V, _V, _V, _V, _L, _D, _D, _D, _D, _V, _V, _V, _V, _V, _V],
    "pm_split_positions": [_V, _V, _V, _V, _L, _V, _V, _V, _V],
    "pm_join_positions": [_V, _V, _V, _V, _V, _L, _V, _V, _V],
    "pm_deposit_f32": [_V, _V, _V, _V, _V, _L, _F, _V],
    "pm_sort_f32": [_V, _V, _V, _V, _V, _V, _V, _V, _L],
    "pm_fft_r2c_f32": [_V, _V],
    "pm_green_f32": [_V, _V, _D],
    "pm_fft_c2r_f32": [_V, _V],
    "pm_poisson_f32": [_V, _V, _D],
    "pm_interp_f32": [_V, _V, _V, _V, _V, _V, _L, _V, _V, _V],
    "pm_kick_drift_f32": [_V, _V, _V, _V, _V, _V, _V, _V, _V, _L, _D, _D],
    "pm_step_f32": [_V, _V, _V, _V, _V, _V, _V, _V, _L, _F, _D, _D, _D],
    "pm_potential_f32": [_V, _V, _V, _V, _V, _L, _F, _D],
    "pm_plan_set_fft_shape": [_V, _I, _I],
    "pm_plan_set_gather": [_V, _I],
    "pm_reduce_f32": [_V, _V, _V, _V, _V, _L, _D, _V],
    "pm_reduce_f64": [_V, _V, _V, _V, _V, _L, _D, _V],
    "pm_adjoint_deposit_f32": [_V, _V, _V, _V, _V, _L, _F, _V, _V, _V, _V],
    "pm_adjoint_force_f32": [_V, _V, _V, _V, _V, _L, _F, _D, _V, _V, _V, _D, _V, _V, _V],
    "pm_step_adjoint_f32": [_V, _V, _V, _V, _V, _L, _F, _D, _D, _D, _V, _V, _V, _V, _V, _V],
    "pm_deposit_f32_noalloc": [_I, _V, _V, _V, _V, _L, _F, _V, _V],
    "pm_ensemble_create": [_I, _V, _V, _V, _I, _I, _I, ctypes.c_char_p, _V, ctypes.POINTER(_V)],
    "pm_ensemble_destroy": [_V],
    "pm_ensemble_sync": [_V],
    "pm_ensemble_step_f32": [_V, _V, _V, _V, _V, _V, _V, _V, _D, _D, _D],
    "pm_ensemble_run_f32": [_V, _V, _V, _V, _V, _V, _V, _V, _D, _D, _I],
    "pm_ensemble_info": [_V, _V, _V, _V, _V, _V, _V, _V],
    "pm_ic_zeldovich": [_I, _I, _D, _D, _U64, _D, _V, _V, _V, _V, _V, _V, _V],
    "pm_slab_create": [_I, _I, _I, _I, _I, _V, ctypes.POINTER(_V)],
    "pm_slab_destroy": [_V],
    "pm_slab_info": [_V, _V, _V, _V, _V, _V, _V, _V, _V],
    "pm_slab_plan": [_V, ctypes.POINTER(_V)],
    "pm_slab_deposit_f32": [_V, _V, _V, _V, _V, _L, _F],
    "pm_slab_fold_f32": [_V, _V],
    "pm_slab_forward_f32": [_V],
    "pm_slab_xgreen_f32": [_V, _D],
    "pm_slab_backward_f32": [_V],
    "pm_slab_kick_drift_f32": [_V, _V, _V, _V, _V, _V, _V, _V, _L, _D, _D],
    "pm_slab_migrate_sort": [_V, _V, _L, _V],
    "pm_slab_migrate_pack": [_V, _V, _I, _L, _V],
    "pm_slab_migrate_unpack": [_V, _V, _L, _V, _I, _L],
    "pm_slab_check": [_V],
    "pm_ipc_export": [_V, _V],
    "pm_ipc_open": [_V, ctypes.POINTER(_V)],
    "pm_ipc_close": [_V],
    "pm_slab_forward_peers_f32": [_V, _V, _I],
    "pm_slab_xgreen_peers_f32": [_V, _V, _D, _V, _I],
    "pm_slab_backward_rows_f32": [_V, _V],
    "pm_pencil_create": [_I, _I, _I, _I, _I, _I, _V, ctypes.POINTER(_V)],
    "pm_pencil_destroy": [_V],
    "pm_pencil_info": [_V, _V, _V, _V, _V, _V, _V, _V, _V, _V],
    "pm_pencil_plan": [_V, ctypes.POINTER(_V)],
    "pm_pencil_deposit_f32": [_V, _V, _V, _V, _V, _L, _F],
    "pm_pencil_fold_f32": [_V, _V, _V, _V],
    "pm_pencil_forward_f32": [_V],
    "pm_pencil_yfwd_f32": [_V],
    "pm_pencil_xgreen_f32": [_V, _D],
    "pm_pencil_yinv_f32": [_V],
    "pm_pencil_backward_f32": [_V],
    "pm_pencil_kick_drift_f32": [_V, _V, _V, _V, _V, _V, _V, _V, _L, _D, _D],
    "pm_pencil_migrate_sort": [_V, _V, _L, _V],
    "pm_pencil_migrate_pack": [_V, _V, _I, _L, _V],
    "pm_pencil_migrate_unpack": [_V, _V, _L, _V, _I, _L],
    "pm_pencil_check": [_V],
    "pm_pencil_forward_peers_f32": [_V, _V, _I],
    "pm_pencil_yfwd_peers_f32": [_V, _V, _V, _I],
    "pm_pencil_xgreen_peers_f32": [_V, _V, _D, _V, _I],
    "pm_pencil_yinv_peers_f32": [_V, _V, _V, _I],
    "pm_pencil_backward_from_f32": [_V, _V],
}

_lib = None


class PMError(RuntimeError):
    """A C-ABI call returned a status other than PM_OK."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{_STATUS.get(code, code)}: {msg}")
        self.code = code


def header_symbols() -> list[str]:
    """Function names declared in include/pm_b200.h."""
    import re
    path = os.path.join(os.path.dirname(HERE), "include", "pm_b200.h")
    with open(path) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(pm_\w+)\s*\(", text, re.M)))


STAGE_COUNT = 19


def load(build_if_missing: bool = True) -> ctypes.CDLL:
    """Loads libpm_b200.so (building it with nvcc if absent or stale)."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing:
        import importlib.util
        spec = importlib.util.spec_from_file_location("_pm_b200_build", os.path.join(HERE, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        try:
            mod.build()
        except Exception as e:  # noqa: BLE001 -- no nvcc: use the library if it exists
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"libpm_b200.so is missing and could not be built: {e}") from e
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} not found (build with particle-mesh_b200/build.py)")
    L = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    L.pm_last_error.argtypes = []
    L.pm_last_error.restype = ctypes.c_char_p
    L.pm_stage_name.argtypes = [_I]
    L.pm_stage_name.restype = ctypes.c_char_p
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != PM_OK:
        raise PMError(rc, load().pm_last_error().decode(errors="replace"))
