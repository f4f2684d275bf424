"""The allocation-free deposit entry point, for callers that cannot allocate
device memory themselves (a host framework's allocator owns every device
allocation, or the per-step path must not allocate).

It is called through the C ABI twice in a row, on different particle sets,
and each result is checked against the allocating pm_deposit_f32 on the same
inputs.  The second call would see the first call's leftovers in the shared
static scratch if the entry point did not clear what must start at zero.
The file sorts last so a stop-at-first-failure run has already run every
other test; it also runs alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = "cuda:0"
TOL = 1e-5  # absolute, on values of order 1 (same tolerance as the FP32 tile-deposit parity test)


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


# (ng, particle counts of the calls in a row): the 16^3-tile kernel at 128;
# the 8^3-tile kernel of the smallest mesh; the largest mesh with a particle
# set that fills the static permutation exactly; and empty sets before and
# after a full one (an empty call must not see the previous call's buckets).
CASES = [(128, (300000, 200000)), (8, (300, 1000)), (256, (1 << 21, (1 << 21) - 12345)),
         (64, (0, 5000, 0))]


@pytest.mark.parametrize("ng,counts", CASES, ids=[f"ng{c[0]}" for c in CASES])
def test_no_alloc_deposit_matches_allocating_entry_point(pmpkg, ng, counts):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = pmpkg.load()
    plan = pmpkg.Plan(ng, "fp32", device=DEV)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for seed, np_ in enumerate(counts, start=1):
        rng = np.random.default_rng(seed + ng)
        pos = [torch.tensor(rng.uniform(0, ng, np_), dtype=torch.float64, device=DEV) for _ in range(3)]
        cell, off = plan.split(*pos)
        mass = 0.37 * seed
        ref = plan.deposit_split(cell, off, mass)
        out = torch.full((ng, ng, ng + 2), float("nan"), dtype=torch.float32, device=DEV)
        rc = lib.pm_deposit_f32_noalloc(ng, _vp(cell), *(_vp(t) for t in off), np_, mass, _vp(out), stream)
        assert rc == 0, lib.pm_last_error()
        torch.cuda.synchronize()
        assert torch.isfinite(out).all()
        assert float((out - ref).abs().max()) < TOL * max(1.0, mass * np_ / ng ** 3 * 8)
        if np_ == 0:
            assert torch.equal(out[:, :, :ng], torch.full_like(out[:, :, :ng], -1.0))
        assert torch.equal(out[:, :, ng:], torch.zeros_like(out[:, :, ng:]))


def test_no_alloc_deposit_rejects_sizes_beyond_its_limits(pmpkg):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = pmpkg.load()
    dummy = torch.zeros(4, dtype=torch.float32, device=DEV)
    p = _vp(dummy)
    assert lib.pm_deposit_f32_noalloc(512, p, p, p, p, 1, 1.0, p, None) == 2  # PM_ERR_SIZE
    assert b"256" in lib.pm_last_error()
    assert lib.pm_deposit_f32_noalloc(64, p, p, p, p, (1 << 21) + 1, 1.0, p, None) == 2
    assert b"2097152" in lib.pm_last_error()
    assert lib.pm_deposit_f32_noalloc(64, None, p, p, p, 1, 1.0, p, None) == 1  # PM_ERR_ARG
