"""The CPU oracle checked against independent references.

The reference ships no tests, fixtures or outputs and cannot be built here
(Fortran, no compiler), so the restatement is pinned by mathematics:
  * FFT/REALTR against numpy's real FFT (exact in -r8 literal mode, and the
    gcc-literal mode's single-precision-angle error quantified);
  * BLKTRI against scipy sparse LU on the same block-tridiagonal systems,
    including the real POT3 operators with a long-double-refined solution;
  * POT3 against a manufactured solution of its own discrete operator;
  * BDYGEN against multipole known answers;
  * the committed regression fixtures (tests/golden/).
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from chymera_uo_b200 import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# ---------------------------------------------------------------------------
# FFT / REALTR (pot/fft.f)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n", [2, 4, 8, 16, 32, 64, 128, 256, 512])
def test_fft_matches_numpy_exp_plus(ora, n):
    """FFT(A,B,N,N,N,+1) is the exp(+i) DFT (pot/fft.f:91-92)."""
    rng = np.random.default_rng(n)
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    A, B = a.copy(), b.copy()
    ora.fft(A, B, 1, True)
    ref = np.fft.ifft(a + 1j * b) * n
    assert np.abs(A + 1j * B - ref).max() <= 1e-13 * np.abs(ref).max()
    A, B = a.copy(), b.copy()
    ora.fft(A, B, -1, True)
    ref = np.fft.fft(a + 1j * b)
    assert np.abs(A + 1j * B - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("L", [32, 64, 128, 256, 512])
def test_realtr_r8_equals_rfft(ora, L):
    """POT3's forward transform with -r8 literals: cosine coefficients
    Re(rfft)/N and sine coefficients -Im(rfft)/N (pot/pot3.f:95-140)."""
    x = np.random.default_rng(L).standard_normal(L)
    m = ora.forward_real(x, True)
    n = L // 2
    ref = np.fft.rfft(x)
    assert np.abs(m[: n + 1] - ref.real / n).max() < 1e-14 * np.abs(x).max() * 4
    assert np.abs(m[n + 1:] + ref.imag[1:n] / n).max() < 1e-14 * np.abs(x).max() * 4


@pytest.mark.parametrize("L", [64, 128, 256])
def test_gcc_literal_transform_differs_by_single_precision_pi(ora, L):
    """gcc-literal builds take the twiddle angle from REAL(4) ATAN(1.0)
    (pot/fft.f:38,129): the transform differs from the exact DFT at ~1e-7.
    The -r8 pair round-trips to rounding; the gcc pair does only when every
    stage is radix 4 (LMAX = 128): radix-2 stages rotate the partner of
    position j by the true pi (pot/fft.f:221-224), so the gcc forward and
    inverse transforms are not exact inverses -- which is why refinement has to
    work on the mode-space equations."""
    x = np.random.default_rng(7).standard_normal(L)
    g = ora.forward_real(x, False)
    r = ora.forward_real(x, True)
    rel = np.abs(g - r).max() / np.abs(r).max()
    assert 1e-9 < rel < 1e-6
    assert np.abs(ora.inverse_real(r, True) - x).max() < 1e-14 * 8
    rt = np.abs(ora.inverse_real(g, False) - x).max()
    if L == 128:
        assert rt < 1e-14 * 8
    else:
        assert 1e-10 < rt < 1e-6


# ---------------------------------------------------------------------------
# BLKTRI (pot/blktri.f)
# ---------------------------------------------------------------------------
def _assemble(an, bn, cn, am, bm, cm):
    M, N = len(am), len(an)
    Tm = sp.diags([am[1:], bm, cm[:-1]], [-1, 0, 1])
    Tn = sp.diags([an[1:], bn, cn[:-1]], [-1, 0, 1])
    return (sp.kron(Tn, sp.eye(M)) + sp.kron(sp.eye(N), Tm)).tocsc()


@pytest.mark.parametrize("M,N", [(15, 7), (63, 31), (255, 127)])
def test_blktri_random_systems(ora, M, N):
    rng = np.random.default_rng(M)
    an, cn = rng.uniform(0.5, 1.5, N), rng.uniform(0.5, 1.5, N)
    bn = -(an + cn) - rng.uniform(0, 1, N)
    an[0] = cn[-1] = 0
    am, cm = rng.uniform(0.5, 1.5, M), rng.uniform(0.5, 1.5, M)
    bm = -(am + cm) - rng.uniform(0, 1, M)
    am[0] = cm[-1] = 0
    y = rng.standard_normal((M, N))
    x, ierr = ora.blktri_solve(an, bn, cn, am, bm, cm, y.copy(order="F"))
    assert ierr == 0
    xs = spl.spsolve(_assemble(an, bn, cn, am, bm, cm), y.flatten(order="F")).reshape((M, N), order="F")
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-13


def test_blktri_error_codes(ora):
    """IERROR 2: N not 2**k-1 (pot/blktri.f:29-31)."""
    M, N = 15, 6
    an = np.ones(N); cn = np.ones(N); bn = -3 * np.ones(N)
    am = np.ones(M); cm = np.ones(M); bm = -3 * np.ones(M)
    _, ierr = ora.blktri_solve(an, bn, cn, am, bm, cm, np.zeros((M, N), order="F"))
    assert ierr == 2


def pot3_operator(J, K, L, m, lit=False):
    """POT3's mode-m operator coefficients (pot/pot3.f:158-230), numpy."""
    g = synth.default_grid(J, K, L)
    rhf, zhf = g.rhf(), g.zhf()
    RHF = lambda j: rhf[j - 1]
    ZHF = lambda k: zhf[k - 1]
    dth = g.dtheta
    rd2 = np.zeros(J + 1); rd3 = np.zeros(J + 1); den = np.zeros(J + 1)
    rd2[1] = 0.5 / RHF(2); rd3[1] = 1.0 / RHF(1)
    for j in range(2, J + 1):
        den[j] = 1.0 / (RHF(j + 1) - RHF(j - 1)); rd2[j] = 1.0 / (RHF(j + 1) - RHF(j)); rd3[j] = 1.0 / RHF(j)
    zd2 = np.zeros(K + 1); dz = np.zeros(K + 1)
    zd2[1] = 0.5 / ZHF(2)
    for k in range(2, K + 1):
        dz[k] = 1.0 / (ZHF(k + 1) - ZHF(k - 1)); zd2[k] = 1.0 / (ZHF(k + 1) - ZHF(k))
    cm = np.array([2. * (rd2[j] + 0.5 * rd3[j]) * den[j] for j in range(2, J + 1)])
    am = np.array([2. * (rd2[j - 1] - 0.5 * rd3[j]) * den[j] for j in range(2, J + 1)])
    c = np.array([rd3[j] * rd3[j] / (dth * dth) for j in range(2, J + 1)])
    cn = np.array([2. * zd2[k] * dz[k] for k in range(2, K + 1)])
    an = np.array([2. * zd2[k - 1] * dz[k] for k in range(2, K + 1)])
    bn = -cn - an
    cmmax, ammin, cnmax = cm[-1], am[0], cn[-1]
    cm[-1] = 0; am[0] = 0; cn[-1] = 0; bn[0] = -cn[0]; an[0] = 0
    xl = np.cos(m * dth)
    bm = -cm - am + 2 * (xl - 1) * c
    bm[0] = -cm[0] + ((-1.0) ** m - 1) * ammin + 2 * (xl - 1) * c[0]
    bm[-1] = -cmmax - am[-1] + 2 * (xl - 1) * c[-1]
    return dict(an=an, bn=bn, cn=cn, am=am, bm=bm, cm=cm, c=c, cmmax=cmmax, ammin=ammin, cnmax=cnmax)


@pytest.mark.parametrize("m", [0, 1, 16, 128])
def test_blktri_pot3_operator_accuracy(ora, m):
    """On the 256x128 POT3 operators BLKTRI agrees with a long-double
    refined sparse solution.  Its own error is largest for the m=0 mode
    (about 2.4e-12 relative L2): the floor any FP64 reimplementation is
    compared against."""
    J, K = 256, 128
    op = pot3_operator(J, K, 256, m)
    M, N = J - 1, K - 1
    jj = np.arange(M)[:, None]; kk = np.arange(N)[None, :]
    y = np.exp(-((jj - 40) / 30.0) ** 2 - (kk / 20.0) ** 2) * (1 + 0.1 * np.random.default_rng(0).standard_normal((M, N)))
    A = _assemble(op["an"], op["bn"], op["cn"], op["am"], op["bm"], op["cm"])
    lu = spl.splu(A)
    b = y.flatten(order="F")
    x = lu.solve(b)
    Al = A.astype(np.longdouble)
    for _ in range(3):
        r = b.astype(np.longdouble) - Al @ x.astype(np.longdouble)
        x = x + lu.solve(r.astype(np.float64))
    xt = x.reshape((M, N), order="F")
    xb, ierr = ora.blktri_solve(op["an"], op["bn"], op["cn"], op["am"], op["bm"], op["cm"], y.copy(order="F"))
    assert ierr == 0
    err = np.linalg.norm(xb - xt) / np.linalg.norm(xt)
    assert err < 5e-12


# ---------------------------------------------------------------------------
# POT3 against a manufactured solution of its discrete operator
# ---------------------------------------------------------------------------
def apply_pot3_operator(phi, J, K, L):
    """The real-space 7-point operator POT3 inverts (pot/pot3.f:158-230),
    applied to a full PHI array: radial AM/CM, vertical AN/CN, azimuthal
    C(J)(PHI(L+1) - 2 PHI(L) + PHI(L-1)), the axis ghost PHI(1,K,L) =
    PHI(2,K,L+N), the midplane ghost PHI(J,1,L) = PHI(J,2,L), Dirichlet
    values at J = JMAX+1 and K = KMAX+1.  Returns A(phi) on the interior."""
    op = pot3_operator(J, K, L, 0)
    N = L // 2
    M, NZ = J - 1, K - 1
    P = phi[1:J, 1:K, :]                       # interior (j=2..J, k=2..K)
    out = np.zeros_like(P)
    am = np.r_[op["ammin"], op["am"][1:]][:, None, None]
    cmr = np.r_[op["cm"][:-1], op["cmmax"]][:, None, None]
    up = np.concatenate([phi[2:J + 1, 1:K, :]], axis=0)         # j+1 (J+1 is the boundary)
    axis = np.roll(phi[1:2, 1:K, :], -N, axis=2)                # PHI(2,K,L+N)
    down = np.concatenate([axis, phi[1:J - 1, 1:K, :]], axis=0)  # j-1
    out += am * down + cmr * up - (am + cmr) * P
    c = op["c"][:, None, None]
    out += c * (np.roll(P, -1, axis=2) - 2 * P + np.roll(P, 1, axis=2))
    an = np.r_[0.0, op["an"][1:]][None, :, None]
    cnr = np.r_[op["cn"][:-1], op["cnmax"]][None, :, None]
    zup = phi[1:J, 2:K + 1, :]
    zdn = np.concatenate([phi[1:J, 1:2, :], phi[1:J, 1:K - 1, :]], axis=1)   # midplane ghost = PHI(J,2)
    cn0 = op["cn"][0]
    anr = np.r_[cn0, op["an"][1:]][None, :, None]   # at k=1 the ghost term uses CN(1)
    out += anr * zdn + cnr * zup - (anr + cnr) * P
    return out


def test_pot3_manufactured_solution(ora):
    """With -r8 literals POT3 inverts its 7-point operator exactly: choose
    PHI, set RHO = A(PHI)/(4 pi G) and the Dirichlet boundary values, run
    POT3 alone, and recover PHI."""
    J, K, L = 32, 16, 32
    g = synth.default_grid(J, K, L)
    r = g.rhf()[:, None, None]; z = g.zhf()[None, :, None]
    psi = ((np.arange(L) + 0.5) * g.dtheta)[None, None, :]
    phi = (np.exp(-(r ** 2 + z ** 2)) * (1 + 0.3 * np.cos(2 * psi) * r ** 2 + 0.1 * np.sin(3 * psi) * r ** 3)
           ).astype(np.float64)
    phi = np.asfortranarray(phi)
    A = apply_pot3_operator(phi, J, K, L)
    o = ora.Oracle(J, K, L, literal_r8=True)
    o.set_grid(1.0 / J, 0.5 / K)
    rho = np.zeros((J + 2, K + 2, L), order="F")
    rho[1:J, 1:K, :] = A / (4.0 * np.pi)
    o.rho[...] = rho
    o.phi[...] = 0.0
    o.phi[J, 1:K + 1, :] = phi[J, 1:K + 1, :]     # outer boundary J = JMAX+1
    o.phi[1:J + 1, K, :] = phi[1:J + 1, K, :]     # top boundary K = KMAX+1
    o.pot3(8, 0)
    got = np.array(o.phi)
    err = np.abs(got[1:J, 1:K, :] - phi[1:J, 1:K, :]).max() / np.abs(phi).max()
    assert err < 1e-12


# ---------------------------------------------------------------------------
# BDYGEN multipole known answers (pot/boundary.f)
# ---------------------------------------------------------------------------
def _boundary_values(ora, rho, J, K, L, **kw):
    o = ora.Oracle(J, K, L)
    o.set_grid(1.0 / J, 0.5 / K)
    o.rho[...] = rho
    o.phi[...] = 0.0
    o.setbdy(0, kw.get("isym", 2))
    assert o.bdygen(kw.get("maxtrm", 10), kw.get("isym", 2), 0.0) == 0
    return np.array(o.phi), o.inside(), np.array(o.rbdy)


def test_bdygen_compact_mass_is_monopole(ora):
    """A compact mass near the origin gives PHI ~ -G M / r on the boundary."""
    J, K, L = 64, 32, 64
    rho = np.zeros((J + 2, K + 2, L), order="F")
    rho[1:3, 1:3, :] = 1.0
    phi, d, rb = _boundary_values(ora, rho, J, K, L)
    top = phi[1:J + 1, K, 0]
    rtop = rb[:J]
    assert np.allclose(top, -d["tmass"] / rtop, rtol=2e-3)


def test_bdygen_axisymmetric_density_gives_axisymmetric_boundary(ora):
    J, K, L = 64, 32, 64
    rho = synth.disk_density(J, K, L, 5, noise=0.0)
    phi, _, _ = _boundary_values(ora, rho, J, K, L)
    top = phi[1:J + 1, K, :]
    assert np.abs(top - top[:, :1]).max() <= 1e-13 * np.abs(top).max()


def test_bdygen_pure_azimuthal_mode(ora):
    """rho = rho0(r,z) (1 + eps cos 3 psi) puts boundary power only in m = 0, 3."""
    J, K, L = 64, 32, 64
    base = synth.disk_density(J, K, L, 5, noise=0.0)
    psi = (np.arange(1, L + 1) - 0.5) * 2 * np.pi / L
    rho = np.asfortranarray(base * (1 + 0.2 * np.cos(3 * psi))[None, None, :])
    phi, _, _ = _boundary_values(ora, rho, J, K, L)
    spec = np.abs(np.fft.rfft(phi[1:J + 1, K, :], axis=1)).max(axis=0)
    others = np.delete(spec, [0, 3])
    assert others.max() < 1e-10 * spec[3]


# ---------------------------------------------------------------------------
# Regression fixtures
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["disk_32x16x32_gcc", "disk_32x16x32_r8", "disk_32x16x32_isym1_m8_np7"])
def test_oracle_matches_fixture(ora, name):
    f = np.load(os.path.join(GOLDEN, name + ".npz"))
    J, K, L = int(f["J"]), int(f["K"]), int(f["L"])
    rho = synth.disk_density(J, K, L, int(f["seed"]), spiral=True, spectrum=True)
    o = ora.Oracle(J, K, L, literal_r8=bool(f["r8"]))
    phi = o.solve(rho, isym=int(f["isym"]), maxtrm=int(f["maxtrm"]), redge=float(f["redge"]),
                  npoint=int(f["npoint"]))
    assert np.array_equal(phi, f["phi"])
    d = o.inside()
    assert d["tmass"] == float(f["tmass"]) and d["klocat"] == int(f["klocat"])


def test_oracle_threads_agree_with_serial(ora):
    """The OpenMP merge order changes BDYGEN's sums only at rounding level."""
    rho, g = synth.config_density(1)
    p1 = ora.Oracle(64, 32, 64, nthreads=1).solve(rho)
    p4 = ora.Oracle(64, 32, 64, nthreads=4).solve(rho)
    assert np.linalg.norm(p4 - p1) / np.linalg.norm(p1) < 1e-13


# ---------------------------------------------------------------------------
# ExternalPot (pot/ExternalPot.f:1-80)
# ---------------------------------------------------------------------------
def _starphi_scalar(rhf, zhf, L, dtheta, mass, ix, iy):
    """pot/ExternalPot.f:44-49 term by term with Python floats (libm cos/sin)."""
    import math
    out = np.zeros((len(rhf), len(zhf), L), order="F")
    for l in range(1, L + 1):
        c = math.cos((float(l - 1) + 0.5) * dtheta)
        s = math.sin((float(l - 1) + 0.5) * dtheta)
        for k, z in enumerate(zhf):
            for j, r in enumerate(rhf):
                out[j, k, l - 1] = -mass / math.sqrt(r * r + z * z + ix * ix + iy * iy - 2.0 * r * (c * ix + s * iy))
    return out


def test_external_pot_centred_star_is_point_mass(ora):
    J, K, L = 16, 8, 16
    o = ora.Oracle(J, K, L)
    o.set_grid(1.0 / J, 0.5 / K)
    before = np.array(o.phi)
    sp, (ix, iy) = o.external_pot(mass_star=1.0, tmassacc=0.25)
    assert ix == 0.0 and iy == 0.0
    R, Z = np.meshgrid(o.rhf, o.zhf, indexing="ij")
    want = -1.25 / np.sqrt(R * R + Z * Z)
    assert np.array_equal(sp, np.repeat(want[:, :, None], L, axis=2))
    assert np.array_equal(o.phi, before + sp)


def test_external_pot_offset_star_term_by_term(ora):
    import math
    J, K, L = 8, 4, 8
    o = ora.Oracle(J, K, L)
    o.set_grid(1.0 / J, 0.5 / K)
    rng = np.random.default_rng(3)
    o.phi[...] = rng.standard_normal(o.phi.shape)
    before = np.array(o.phi)
    sp, (ix, iy) = o.external_pot(mass_star=0.9, tmassacc=0.01, rpstar=0.013, phi_star=2.1)
    assert ix == 0.013 * math.cos(2.1) and iy == 0.013 * math.sin(2.1)
    want = _starphi_scalar(o.rhf, o.zhf, L, 2.0 * 3.1415926535897932 / L, 0.9 + 0.01, ix, iy)
    assert np.array_equal(sp, want)
    assert np.array_equal(o.phi, before + sp)
    # the potential is lowest at the cell nearest the star
    assert np.isfinite(sp).all() and (sp < 0).all()


def test_external_pot_indirect_shift(ora):
    import math
    J, K, L = 16, 8, 16
    o = ora.Oracle(J, K, L)
    o.set_grid(1.0 / J, 0.5 / K)
    rho = synth.disk_density(J, K, L, 2, spiral=True, spectrum=True)
    o.rho[...] = rho
    dth = 2.0 * 3.1415926535897932 / L
    for jmin in (1, 2, 7):
        _, (ix, iy) = o.external_pot(mass_star=2.0, rpstar=0.01, phi_star=0.3, indirect=True, jmin=jmin)
        psi = (np.arange(L) + 0.5) * dth
        sub = rho[jmin - 1:J + 1, 1:K + 1, :]
        r = np.asarray(o.rhf[jmin - 1:J + 1])[:, None, None]
        m = sub * r * (1.0 / J) * (0.5 / K) * 2.0 * dth
        sx = float(np.sum(m * np.cos(psi) * r))
        sy = float(np.sum(m * np.sin(psi) * r))
        assert ix == pytest.approx(-(0.01 * math.cos(0.3) + sx) / 2.0, rel=1e-13)
        assert iy == pytest.approx(-(0.01 * math.sin(0.3) + sy) / 2.0, rel=1e-13)


# ---------------------------------------------------------------------------
# SOURCE's potential, pressure and rotation terms (radhydro/source.f:45-81)
# ---------------------------------------------------------------------------
def test_source_terms_match_numpy_and_conserve(ora):
    """The oracle's S, T, A updates against a numpy statement of the same
    differences (exact in this order of operations), and the A update's sum
    over L of the pressure part vanishes (periodic differences)."""
    J, K, L = 12, 6, 8
    rng = np.random.default_rng(4)
    hs = (J + 2, K + 2, L)
    rho, phi, omega, p = (np.asfortranarray(rng.random(hs)) for _ in range(4))
    s, t, a = (np.asfortranarray(rng.random(hs)) for _ in range(3))
    s0, t0, a0 = s.copy(), t.copy(), a.copy()
    r = (np.arange(1, J + 3) - 2) * 0.1
    dr, dz, dth, delt = 0.1, 0.05, 2 * np.pi / L, 1e-3
    ora.source(r, rho, phi, omega, p, s, t, a, delt, dr, dz, dth, jmin=2)
    j = slice(2, J + 1)          # J = 3..JMAX1 (0-based 2..J)
    jm = slice(1, J)
    k = slice(1, K + 1)
    rs = rho[j, k] + rho[jm, k]
    om = omega[j, k] + omega[jm, k]
    want_s = s0[j, k] + delt * (r[j, None, None] * rs * (om * om) * 0.25 * 0.5 -
                                rs * (phi[j, k] - phi[jm, k]) / (2 * dr) - (p[j, k] - p[jm, k]) / dr)
    assert np.array_equal(s[j, k], want_s)
    jj = slice(1, J + 1)
    km = slice(0, K)
    want_t = t0[jj, k] - delt * (0.5 * (rho[jj, k] + rho[jj, km]) * (phi[jj, k] - phi[jj, km]) / dz +
                                 (p[jj, k] - p[jj, km]) / dz)
    assert np.array_equal(t[jj, k], want_t)
    lp, lm = np.roll(np.arange(L), -1), np.roll(np.arange(L), 1)
    want_a = a0[jj, k] - delt * (rho[jj, k] * (phi[jj, k][:, :, lp] - phi[jj, k][:, :, lm]) +
                                 p[jj, k][:, :, lp] - p[jj, k][:, :, lm]) / (2 * dth)
    assert np.array_equal(a[jj, k], want_a)
    # untouched: J = 1 and 2 of S, K = 1 and KMAX+2 everywhere
    assert np.array_equal(s[:2], s0[:2]) and np.array_equal(t[:, 0], t0[:, 0])
    assert np.array_equal(a[:, K + 1], a0[:, K + 1])


def test_source_binary_terms_match_numpy(ora):
    """The BINARY build's terms (radhydro/source.f:61-62, 76-77): the oracle's
    S and A against numpy statements of the same left-to-right products,
    added after the BINARY = 0 update of the same statement; T unchanged."""
    import math
    J, K, L = 12, 6, 8
    rng = np.random.default_rng(6)
    hs = (J + 2, K + 2, L)
    rho, phi, omega, p, u = (np.asfortranarray(rng.random(hs)) for _ in range(5))
    s, t, a = (np.asfortranarray(rng.random(hs)) for _ in range(3))
    r = (np.arange(1, J + 3) - 2) * 0.1
    rhf = r + 0.05
    dr, dz, dth, delt = 0.1, 0.05, 2 * np.pi / L, 1e-3
    plain = [x.copy(order="F") for x in (s, t, a)]
    ora.source(r, rho, phi, omega, p, *plain, delt, dr, dz, dth, jmin=3)
    ora.source(r, rho, phi, omega, p, s, t, a, delt, dr, dz, dth, jmin=3,
               binary=dict(mass_star=1.0, mass_bin=0.5, a_bin=1.5, rhf=rhf, u=u))
    mu = 0.5 + 1.0
    ob = math.sqrt(mu / (1.5 * 1.5 * 1.5))      # getBinaryPosition (ExternalRoutines.f:101-102)
    k = slice(1, K + 1)
    j = slice(3, J + 1)          # S: J = JSTART+1..JMAX1 with JSTART = 3
    want_s = plain[0][j, k] + ob * omega[j, k] * rhf[j, None, None] * 2.0 * rho[j, k] * delt
    assert np.array_equal(s[j, k], want_s)
    jj = slice(2, J + 1)         # A: J = JSTART..JMAX1
    want_a = plain[2][jj, k] - rho[jj, k] * ob * (u[3:J + 2, k] + u[jj, k]) * delt * rhf[jj, None, None]
    assert np.array_equal(a[jj, k], want_a)
    assert np.array_equal(t, plain[1])
    # cells outside the loops are the BINARY = 0 build's
    assert np.array_equal(s[:3], plain[0][:3]) and np.array_equal(a[:2], plain[2][:2])
