"""The gfortran-callable SETBDY / BDYGEN / POT3 shims over the reference's
COMMON blocks (chymera_uo_b200/csrc/compat/pot3_common.cpp), driven by a C
program that lays the COMMON blocks out as a gfortran executable does
(tests/compat/harness.c) and issues the ITYPE=71 call sequence of
radhydro/io.f:212-218.  The CPU test compiles and links it; the GPU test runs
it against the oracle (PHI rel. L2 <= 1e-12 over the write set, /INSIDE/,
/COEFS/)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
J, K, L = 64, 32, 64


def build_harness(tmp):
    """Compiles the shim for J x K x L and links the harness; returns the path."""
    dims = [f"JMAX={J}", f"KMAX={K}", f"LMAX={L}"]
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "chymera_uo_b200", "csrc", "compat"), f"OUT={tmp}"]
                   + dims, check=True)
    obj = os.path.join(tmp, f"pot3_common_{J}x{K}x{L}.o")
    hobj = os.path.join(tmp, "harness.o")
    subprocess.run(["gcc", "-O2", "-std=c11", f"-DCHY_JMAX={J}", f"-DCHY_KMAX={K}", f"-DCHY_LMAX={L}", "-c",
                    os.path.join(ROOT, "tests", "compat", "harness.c"), "-o", hobj], check=True)
    exe = os.path.join(tmp, "harness")
    libdir = os.path.join(ROOT, "chymera_uo_b200")
    subprocess.run(["g++", hobj, obj, "-o", exe, f"-L{libdir}", "-lchy_pot3", f"-Wl,-rpath,{libdir}", "-lm"],
                   check=True)
    return exe, obj


def test_shims_compile_and_link(chylib, tmp_path):
    exe, obj = build_harness(str(tmp_path))
    assert os.path.exists(exe)
    syms = subprocess.run(["nm", obj], capture_output=True, text=True, check=True).stdout
    for name in ("setbdy_", "bdygen_", "pot3_", "chy_compat_status_"):
        assert f" T {name}" in syms, name
    for common in ("pois_", "grid_", "blok6_", "inside_", "coefs_"):
        assert f" U {common}" in syms, common      # bound to the program's COMMON blocks


@pytest.mark.gpu
def test_itype71_sequence_through_common_blocks(chylib, tmp_path):
    from chymera_uo_b200 import synth
    from oracle import oracle as O
    exe, _ = build_harness(str(tmp_path))
    rho = synth.disk_density(J, K, L, 1)
    rho_path = os.path.join(str(tmp_path), "rho.bin")
    rho.ravel(order="F").tofile(rho_path)
    prefix = os.path.join(str(tmp_path), "out")
    r = subprocess.run([exe, rho_path, prefix], capture_output=True, text=True)
    assert r.returncode == 0 and "status 0" in r.stdout, r.stdout + r.stderr
    shape = (J + 2, K + 2, L)
    phi = np.fromfile(prefix + ".phi").reshape(shape, order="F")
    tmass, phichk, klocat = np.fromfile(prefix + ".inside")
    coef = np.fromfile(prefix + ".coef").reshape((J + 2, K + 2, L // 2, 2), order="F")

    o = O.Oracle(J, K, L, nthreads=4, want_coef=True)
    ref = o.solve(rho)
    dref = o.inside()
    cref = np.array(o.coef)
    ws = (slice(0, J + 1), slice(0, K + 1))
    assert np.linalg.norm((phi[ws] - ref[ws]).ravel()) <= 1e-12 * np.linalg.norm(ref[ws].ravel())
    assert np.all(phi[:, K + 1, :] == 0.0) and np.all(phi[J + 1, 0, :] == 0.0)
    assert abs(tmass - dref["tmass"]) <= 1e-13 * dref["tmass"]
    assert int(klocat) == dref["klocat"]
    sel = (slice(1, J + 1), slice(1, K + 1))
    amp, amp_r = coef[sel + (slice(None), 0)], cref[sel + (slice(None), 0)]
    assert np.abs(amp - amp_r).max() <= 1e-9 * np.abs(amp_r).max()

    r = subprocess.run([exe, rho_path, prefix, "nosetup"], capture_output=True, text=True)
    assert r.returncode == 0 and "status 13 13" in r.stdout, r.stdout + r.stderr
