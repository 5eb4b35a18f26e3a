"""The ITYPE=71 driver (chymera_uo_b200/csrc/cli/itype71.cpp): fort.5 and the
list-directed fort.2 of radhydro/io.f:100-166 in, phi3d.NNNNNN out as
gfortran unformatted records (io.f:221-226).  The CPU tests check the input
parsing (repeat counts, D exponents, the density floor) with --check-input;
the GPU test compares PHI with the oracle at rel. L2 <= 1e-12."""
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "chymera_uo_b200", "chy_itype71")
J, K, L, HJ, HK = 64, 32, 64, 70, 40
DELR, DELZ, DENCEN = 1.0 / 64, 0.5 / 32, 2.5


def _denny():
    """An axisymmetric hscf-like density on the (HJ+2, HK+2) grid, with a
    block of exact zeros (written with a repeat count) below the floor."""
    j = np.arange(HJ + 2)[:, None]
    k = np.arange(HK + 2)[None, :]
    r = (j - 1.5) * DELR
    z = (k - 1.5) * DELZ
    d = DENCEN * np.exp(-((r / 0.6) ** 2)) * np.exp(-((z / 0.08) ** 2))
    d[:, 30:] = 0.0
    return d


def write_inputs(dirname, itype=71, itstop=12):
    with open(os.path.join(dirname, "fort.5"), "w") as f:
        f.write("          1.0E0      1.5E0\n      1.666666666666667E0 \n")
        f.write(" ".join(f"{v:06d}" for v in (1, itstop, 2, 3, itype, 1, 6, 0)) + " \n")
        f.write("          9.0e0\t     0.0e0\n")
    d = _denny()
    flat = d.ravel(order="F")
    toks, i = [], 0
    while i < flat.size:
        if flat[i] == 0.0:
            n = 1
            while i + n < flat.size and flat[i + n] == 0.0:
                n += 1
            toks.append(f"{n}*0.0D0")
            i += n
        else:
            toks.append(repr(float(flat[i])).replace("e", "D"))
            i += 1
    with open(os.path.join(dirname, "fort.2"), "w") as f:
        f.write(f" 1.5D0, 0.1, 1.0, 0.3, {DENCEN!r}, 0.2, {DELR!r}, {DELZ!r}, 0.0, 60, 20\n")
        for s in range(0, len(toks), 4):
            f.write("  " + "  ".join(toks[s:s + 4]) + "\n")
    return d


def expected_rho(d):
    rho = np.zeros((J + 2, K + 2, L), order="F")
    core = np.maximum(d[1:J + 1, 1:K + 1], 1e-10 * DENCEN)
    rho[1:J + 1, 1:K + 1, :] = core[:, :, None]
    return rho


def run(tmp, *extra):
    return subprocess.run([EXE, "--dir", str(tmp), "--jmax", str(J), "--kmax", str(K), "--lmax", str(L),
                           "--hj", str(HJ), "--hk", str(HK), *extra], capture_output=True, text=True)


def test_inputs_are_parsed_like_the_reference(chylib, tmp_path):
    d = write_inputs(tmp_path)
    r = run(tmp_path, "--check-input")
    assert r.returncode == 0, r.stderr
    fields = dict(kv.split("=") for kv in r.stdout.split())
    assert fields["ITYPE"] == "71" and fields["ITSTOP"] == "12"
    assert float(fields["ROF3N"]) == DELR and float(fields["DENCEN"]) == DENCEN
    assert fields["JREQ"] == "60" and fields["KZPOL"] == "20"
    assert float(fields["sum(RHO)"]) == pytest.approx(expected_rho(d).sum(), rel=1e-12)


def test_other_itype_is_refused(chylib, tmp_path):
    write_inputs(tmp_path, itype=7)
    r = run(tmp_path, "--check-input")
    assert r.returncode == 2 and "ITYPE is 7" in r.stderr


def read_unformatted(path):
    recs = []
    with open(path, "rb") as f:
        while True:
            head = f.read(4)
            if not head:
                break
            n = struct.unpack("<i", head)[0]
            recs.append(f.read(n))
            assert struct.unpack("<i", f.read(4))[0] == n
    return recs


@pytest.mark.gpu
def test_phi3d_matches_the_oracle(chylib, tmp_path):
    from oracle import oracle as O
    d = write_inputs(tmp_path)
    r = run(tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    recs = read_unformatted(os.path.join(tmp_path, "phi3d.000012"))
    assert len(recs) == 2 and len(recs[0]) == 8 * (J + 2) * (K + 2) * L
    phi = np.frombuffer(recs[0], dtype="<f8").reshape((J + 2, K + 2, L), order="F")
    assert struct.unpack("<d", recs[1])[0] == 0.0
    rho = expected_rho(d)
    ref = O.Oracle(J, K, L, nthreads=4).solve(rho, delr=DELR, delz=DELZ)
    ws = (slice(0, J + 1), slice(0, K + 1))
    assert np.linalg.norm((phi[ws] - ref[ws]).ravel()) <= 1e-12 * np.linalg.norm(ref[ws].ravel())


@pytest.mark.gpu
def test_fort3_holds_the_iprint_report(chylib, tmp_path):
    """The ITYPE=71 branch calls POT3 with IPRINT = 1 before unit 3 is opened
    (radhydro/io.f:208-218, :869): the report goes to fort.3, text equal to
    the reference's edit descriptors applied to the oracle's PHAC and COEF
    (PHAC's values within their printed precision)."""
    from oracle import oracle as O
    from unit3 import check, report
    d = write_inputs(tmp_path)
    r = run(tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    text = open(os.path.join(tmp_path, "fort.3")).read()
    o = O.Oracle(J, K, L, nthreads=4, want_coef=True)
    o.solve(expected_rho(d), delr=DELR, delz=DELZ)
    ref = report(lambda k: o.phac[k - 1], o.coef, J, K, L)
    check(text, ref)
    assert text.startswith("PHAC(1:KMAX1):\n") and text.count(" COEFS=") == J - 1
