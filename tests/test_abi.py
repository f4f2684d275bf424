"""The C ABI library without a GPU: it loads, exports every symbol that
include/pm_b200.h declares, and rejects bad arguments on the host."""
import ctypes

import pytest


@pytest.fixture(scope="module")
def lib(pmpkg):
    return pmpkg.load()


def test_header_symbols_all_exported(pmpkg, lib):
    from particle_mesh_b200 import _lib
    names = _lib.header_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    # and the ctypes table covers the whole header
    assert set(names) - {"pm_last_error", "pm_stage_name"} == set(_lib.SIGNATURES)
    assert lib.pm_stage_name(0) == b"mesh_init" and lib.pm_stage_name(99) == b""


def test_null_arguments_rejected(lib):
    assert lib.pm_plan_create(64, 0, 0, 2, None, None) == 1  # PM_ERR_ARG
    assert b"NULL" in lib.pm_last_error()
    h = ctypes.c_void_p()
    assert lib.pm_plan_create(12, 0, 0, 2, None, ctypes.byref(h)) == 2  # PM_ERR_SIZE
    assert lib.pm_plan_create(64, 7, 0, 2, None, ctypes.byref(h)) == 1
    assert lib.pm_plan_create(64, 0, 0, 3, None, ctypes.byref(h)) == 1
    assert lib.pm_deposit_f64(None, None, None, None, 0, 1.0, None) == 1
    assert lib.pm_step_f32(None, None, None, None, None, None, None, None, 0, 1.0, 1.0, 1.0, 0.0) == 1
    assert lib.pm_plan_check(None) == 1
    assert lib.pm_plan_destroy(None) == 0


def test_plan_create_without_gpu_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    h = ctypes.c_void_p()
    rc = lib.pm_plan_create(64, 0, 0, 2, None, ctypes.byref(h))
    assert rc == 3  # PM_ERR_CUDA
    assert not h.value
    assert lib.pm_last_error()


def test_python_mirror_validates_before_calling(pmpkg):
    import torch
    from particle_mesh_b200 import pm
    with pytest.raises(pmpkg.PMError):
        pm._need(torch.zeros(3), torch.float64, name="x")  # not CUDA
    with pytest.raises(pmpkg.PMError):
        pm._need(torch.zeros(3, dtype=torch.float32), torch.float64, name="x")
