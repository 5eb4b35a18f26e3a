"""Generates the oracle regression fixtures in tests/golden/.

The reference (Fortran CHYMERA) cannot be built here and ships no tests,
fixtures or outputs, so these fixtures pin the oracle to itself: they are the
CPU restatement's PHI and diagnostics for small seeded disks, and guard it
against accidental changes.  Its agreement with the mathematics is tested
separately (numpy FFT, scipy solves, manufactured solutions, multipoles).

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from chymera_uo_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = [
    # name, J, K, L, seed, literal_r8, isym, maxtrm, redge, npoint
    ("disk_32x16x32_gcc", 32, 16, 32, 11, False, 2, 10, 0.0, 8),
    ("disk_32x16x32_r8", 32, 16, 32, 11, True, 2, 10, 0.0, 8),
    ("disk_32x16x32_isym1_m8_np7", 32, 16, 32, 12, False, 1, 8, 0.0, 7),
]


def run_case(J, K, L, seed, r8, isym, maxtrm, redge, npoint):
    rho = synth.disk_density(J, K, L, seed, spiral=True, spectrum=True)
    o = O.Oracle(J, K, L, literal_r8=r8, nthreads=1)
    phi = o.solve(rho, isym=isym, maxtrm=maxtrm, redge=redge, npoint=npoint)
    return rho, phi, o.inside()


def main():
    for name, J, K, L, seed, r8, isym, maxtrm, redge, npoint in CASES:
        rho, phi, d = run_case(J, K, L, seed, r8, isym, maxtrm, redge, npoint)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), phi=phi,
                            tmass=d["tmass"], phichk=d["phichk"], klocat=d["klocat"],
                            J=J, K=K, L=L, seed=seed, r8=r8, isym=isym, maxtrm=maxtrm,
                            redge=redge, npoint=npoint)
        print(name, float(np.abs(phi).max()), d)


if __name__ == "__main__":
    main()
