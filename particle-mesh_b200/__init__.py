"""B200-native particle-mesh step (CUDA kernels for sm_100a behind a C ABI).

The C ABI is include/pm_b200.h (libpm_b200.so, built by build.py); ``pm``
is the Python host side over it, with the reference's stage names.
"""
from . import hostio, pencil, slab  # noqa: F401
from ._lib import PMError, load  # noqa: F401
from .pm import (  # noqa: F401
    DA, FFT, OMEGA_0, Ensemble, OMEGA_K, OMEGA_L, OMEGA_M, START_A, Plan, centered_derivatives, cosmo_run,
    cosmo_schedule, deposit_particles, function_a, read_snapshot, reference_coefficients, unit_box_coefficients,
    update_particles, write_snapshot, zeldovich_ic,
)
