"""Regenerates the golden fixtures in this folder from the reference itself.

Each fixture is one reference step at P = 1 on the reference's own initial
conditions (uniform positions from src/utils/utils.cpp:22-36, seeds 0/1/2,
momenta zero, a = 0.9), computed by the reference's compiled CPU kernels
(oracle/_ref, built from the reference sources by oracle/Makefile), with
numpy.fft standing in for FFTW (not buildable here).  Stored per case:

  pos      (3, np)          input positions, cell units
  mom      (3, np)          momenta after the kick
  delta    (ng, ng, ng)     density contrast after deposit + ghost fold
  phi      (ng, ng, ng)     potential after FFT / Green / inverse FFT
  force    (3, ng, ng, ng)  2-point centred forces (ghost planes dropped)

Run from the repository root on a machine with the reference sources:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

CASES = [(8, 8), (16, 16), (16, 8), (32, 16)]


def make(ng, nrow, full=True):
    x, y, z = O.reference_init_particles(ng, nrow)
    px, py, pz = (np.zeros(nrow ** 3) for _ in range(3))
    mass = float(ng) ** 3 / float(nrow) ** 3
    r = O.reference_force_step(ng, x, y, z, px, py, pz, mass, threads=2)
    out = dict(
        ng=np.int64(ng), nrow=np.int64(nrow), mass=np.float64(mass), a=np.float64(O.START_A),
        pos=np.stack([x, y, z]), mom=np.stack([px, py, pz]),
        delta=np.ascontiguousarray(r["delta"][:, :, :ng]),
    )
    if full:
        out["phi"] = np.ascontiguousarray(r["phi"][:, :, :ng])
        out["force"] = np.stack([f[:ng, :ng, :ng] for f in r["forces"]])
    return out


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    for ng, nrow in CASES:
        d = make(ng, nrow, full=ng <= 16)
        path = os.path.join(here, f"ref_step_ng{ng}_np{nrow}.npz")
        np.savez_compressed(path, **d)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
