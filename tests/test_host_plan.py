"""Host-side parts of libchy_pot3, checked without a GPU: the recorded
transform schedule against the oracle, the plan tables, and the C ABI's
exported symbols and argument checking."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def table(chy, g, name, n):
    out = np.zeros(n)
    m = chy.lib().chy_dbg_table(C.byref(g), name.encode(), dp(out), n)
    assert m >= 0, (name, m)
    return out[:m]


@pytest.mark.parametrize("n", [16, 32, 64, 128, 256, 512])
@pytest.mark.parametrize("isn", [1, -1])
@pytest.mark.parametrize("lit", [0, 1])
def test_recorded_schedule_is_bitwise_the_oracle_fft(chylib, ora, n, isn, lit):
    """The stage/twiddle/permutation tables the device transforms execute,
    applied on the host, reproduce pot/fft.f FFT and REALTR bit for bit."""
    rng = np.random.default_rng(n * 7 + isn + lit)
    a, b = rng.standard_normal(n + 1), rng.standard_normal(n + 1)
    a1, b1, a2, b2 = a.copy(), b.copy(), a.copy(), b.copy()
    assert chylib.lib().chy_dbg_fft(n, isn, lit, dp(a1), dp(b1)) == 0
    ora.fft(a2, b2, isn, bool(lit), n)
    assert np.array_equal(a1[:n], a2[:n]) and np.array_equal(b1[:n], b2[:n])
    a3, b3, a4, b4 = a.copy(), b.copy(), a.copy(), b.copy()
    assert chylib.lib().chy_dbg_realtr(n, isn, lit, dp(a3), dp(b3)) == 0
    ora.realtr(a4, b4, n, isn, bool(lit))
    assert np.array_equal(a3, a4) and np.array_equal(b3, b4)


def test_schedule_rejects_non_power_of_two(chylib):
    a = np.zeros(13); b = np.zeros(13)
    assert chylib.lib().chy_dbg_fft(12, 1, 0, dp(a), dp(b)) == 11   # CHY_ERR_DIMS


@pytest.mark.parametrize("J,K,L", [(64, 32, 64), (256, 128, 256), (128, 64, 128)])
def test_vertical_eigenbasis(chylib, J, K, L):
    g = chylib.grid(J, K, L)
    NZ = K - 1
    U = table(chylib, g, "U", NZ * NZ).reshape(NZ, NZ)
    V = table(chylib, g, "V", NZ * NZ).reshape(NZ, NZ)
    lam = table(chylib, g, "lam", NZ)
    an, bn, cn = table(chylib, g, "an", NZ), table(chylib, g, "bn", NZ), table(chylib, g, "cn", NZ)
    Tz = np.diag(bn) + np.diag(an[1:], -1) + np.diag(cn[:-1], 1)
    assert np.abs(U @ V - np.eye(NZ)).max() < 1e-13
    assert np.abs(V @ np.diag(lam) @ U - Tz).max() < 1e-13 * np.abs(Tz).max()
    assert np.all(lam < 0)   # Neumann midplane + Dirichlet top: negative definite


def test_stencil_matches_pot3_formulas(chylib):
    from tests.test_oracle import pot3_operator
    J, K, L = 64, 32, 64
    g = chylib.grid(J, K, L)
    op = pot3_operator(J, K, L, 0)
    for name in ("an", "bn", "cn", "am", "cm"):
        got = table(chylib, g, name, 256)
        assert np.array_equal(got, op[name]), name
    sc = table(chylib, g, "scalars", 8)
    assert sc[2] == op["cmmax"] and sc[3] == op["ammin"] and sc[4] == op["cnmax"]


@pytest.mark.parametrize("J,K,L", [(64, 32, 64), (80, 32, 64), (256, 128, 32)])
def test_mixed_sweep_table_is_the_two_sided_elimination(chylib, J, K, L):
    """The mixed path's radial sweep table, restated with the same FP64
    operations.  For each m and vertical eigenvalue lam_p (-1 on padding
    rows): the excess g_j = 2 (XLAMM(m) - 1) CC_j, plus the axis term in row
    1 and -CMMAX in row M; rows j < h eliminated top-down
    (t = g_j + lam - AM_j e, 1/D = 1/(t - CM_j), e = t/D), rows j >= h
    bottom-up with AM and CM exchanged, h = 32 ceil(M/64).  The table holds
    the multipliers, then the pivot reciprocals, as FP32 planes [m][j][p]
    with JMAX rounded up to 64 rows; rows past M are zero."""
    g = chylib.grid(J, K, L)
    M, NZ, N, NT = J - 1, K - 1, L // 2, 64 * ((J + 63) // 64)
    h = 32 * ((M + 63) // 64)
    plane = (N + 1) * NT * 128
    tab = table(chylib, g, "sweep", 2 * plane)
    assert tab.size == 2 * plane
    mul = tab[:plane].reshape(N + 1, NT, 128)
    piv = tab[plane:].reshape(N + 1, NT, 128)
    am, cm, cc = (table(chylib, g, n, 4096) for n in ("am", "cm", "cc"))
    xlamm = table(chylib, g, "xlamm", 4096)
    lam = np.full(128, -1.0)
    lam[:NZ] = table(chylib, g, "lam", 4096)
    sc = table(chylib, g, "scalars", 8)
    cmmax, ammin = sc[2], sc[3]
    want_mul = np.zeros((N + 1, NT, 128))
    want_piv = np.zeros((N + 1, NT, 128))
    for m in range(N + 1):
        xl2 = 2.0 * (xlamm[m] - 1.0)
        axis = ((-1.0 if m & 1 else 1.0) - 1.0) * ammin
        gv = xl2 * cc
        gv[0] = axis + gv[0]
        gv[M - 1] = gv[M - 1] - cmmax
        e = np.zeros(128)
        for j in range(h):
            t = (gv[j] + lam) - am[j] * e
            r = 1.0 / (t - cm[j])
            e = t * r
            want_mul[m, j], want_piv[m, j] = e, r
        f = np.zeros(128)
        for j in range(M - 1, h - 1, -1):
            t = (gv[j] + lam) - cm[j] * f
            r = 1.0 / (t - am[j])
            f = t * r
            want_mul[m, j], want_piv[m, j] = f, r
    assert np.array_equal(mul, want_mul.astype(np.float32).astype(np.float64))
    assert np.array_equal(piv, want_piv.astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("J,K,L", [(64, 32, 64), (128, 128, 64)])
def test_mixed_row_scales_symmetrise_the_vertical_operator(chylib, J, K, L):
    """U = Q^T D and V = D^-1 Q with Q orthogonal; the row scales carry d_k,
    1/d_k and the vertical stencil coefficients conjugated by D
    (d_k AN_k / d_(k-1), d_k CN_k / d_(k+1))."""
    g = chylib.grid(J, K, L)
    NZ = K - 1
    Qt = table(chylib, g, "Qt", NZ * NZ).reshape(NZ, NZ)   # Qt[p][k] = Q(k, p)
    d = table(chylib, g, "dsc", NZ)
    U = table(chylib, g, "U", NZ * NZ).reshape(NZ, NZ)
    V = table(chylib, g, "V", NZ * NZ).reshape(NZ, NZ)
    assert np.abs(Qt @ Qt.T - np.eye(NZ)).max() < 1e-13
    assert np.array_equal(U, Qt * d[None, :])
    assert np.array_equal(V, Qt.T / d[:, None])
    z = table(chylib, g, "row_scales", 512).reshape(4, 128)
    an, cn = table(chylib, g, "an", NZ), table(chylib, g, "cn", NZ)
    assert np.array_equal(z[0, :NZ], d) and np.array_equal(z[1, :NZ], 1.0 / d)
    assert np.all(z[0, NZ:] == 1.0) and np.all(z[1, NZ:] == 1.0)
    assert z[2, 0] == 0.0 and np.array_equal(z[2, 1:NZ], d[1:] * an[1:] / d[:-1])
    assert z[3, NZ - 1] == 0.0 and np.array_equal(z[3, :NZ - 1], d[:-1] * cn[:-1] / d[1:])
    assert np.all(z[2:, NZ:] == 0.0)


@pytest.mark.parametrize("J,K,L", [(64, 32, 64), (128, 128, 64)])
def test_mixed_operand_tiles_are_hi_lo_splits(chylib, J, K, L):
    """The eigenbasis operand of the tensor-core products, read back through
    its K-major 128-byte-swizzled layout: hi = fp16(2^12 Q(k,p)) and
    lo = fp16(2^12 Q(k,p) - hi) with rows p and K index k (the tile of Q^T;
    the kernels read its transpose through the MN-major descriptor), zero
    outside NZ x NZ; hi + lo carries 2^12 Q to about 22 bits."""
    g = chylib.grid(J, K, L)
    NZ = K - 1
    tiles = table(chylib, g, "umma_tiles", 2 * 128 * 128).reshape(2, 128, 128)
    Qt = table(chylib, g, "Qt", NZ * NZ).reshape(NZ, NZ)   # Qt[p][k]
    v = 4096.0 * Qt
    hi = v.astype(np.float16).astype(np.float64)
    lo = (v - hi).astype(np.float16).astype(np.float64)
    assert np.array_equal(tiles[0, :NZ, :NZ], hi)
    assert np.array_equal(tiles[1, :NZ, :NZ], lo)
    for q in (0, 1):
        assert not tiles[q, NZ:, :].any() and not tiles[q, :, NZ:].any()
    assert np.max(np.abs(hi + lo - v)) <= 2.0 ** -21 * np.max(np.abs(v))


def test_boundary_splits_are_sorted_ring_counts(chylib):
    """jk_split = number of rings with RSPHER <= RBDY(JK) (pot/boundary.f:561),
    counted on the reference's own FP64 expressions."""
    J, K, L = 64, 32, 64
    g = chylib.grid(J, K, L)
    rs = table(chylib, g, "ring_rsph", (J - 1) * (K - 1))
    split = table(chylib, g, "jk_split", J + K)
    from chymera_uo_b200 import synth
    gg = synth.default_grid(J, K, L)
    rhf, zhf = gg.rhf(), gg.zhf()
    zk2 = zhf[K] * zhf[K]
    rb = [np.sqrt(zk2 + rhf[j - 1] * rhf[j - 1]) for j in range(2, J + 2)]
    rj2 = rhf[J] * rhf[J]
    rb += [np.sqrt(rj2 + zhf[k - 1] * zhf[k - 1]) for k in range(2, K + 1)]
    assert len(split) == len(rb)
    for q, r in enumerate(rb):
        assert split[q] == np.count_nonzero(rs <= r)


def test_rejects_unsupported_grids(chylib):
    out = np.zeros(4)
    for (J, K, L), code in [((64, 48, 64), 2), ((64, 32, 48), 11), ((2, 32, 64), 1)]:
        g = chylib.grid(J, K, L)
        assert chylib.lib().chy_dbg_table(C.byref(g), b"lam", dp(out), 4) == -code
    g = chylib.grid(64, 32, 64, isym=5)
    assert chylib.lib().chy_dbg_table(C.byref(g), b"lam", dp(out), 4) == -12


def _header_functions():
    names = []
    for h in ("chy_pot3.h", "chy_pot3_testing.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(chy_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(chylib):
    names = _header_functions()
    assert "chy_solve" in names and "chy_plan_create" in names
    lib = C.CDLL(chylib.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_argument_checks(chylib):
    L = chylib.lib()
    assert L.chy_status_string(0) == b"ok"
    assert b"BLKTRI IERROR=2" in L.chy_status_string(2)
    p = C.c_void_p()
    assert L.chy_plan_create(None, 0, 1, C.byref(p)) == 10
    g = chylib.grid(64, 32, 64)
    assert L.chy_plan_create(C.byref(g), 7, 1, C.byref(p)) == 10
    assert L.chy_plan_create(C.byref(g), 0, 0, C.byref(p)) == 10
    assert L.chy_solve(None, None, None, None, 0, None) == 10


def test_external_and_source_argument_checks(chylib):
    """The star-potential and SOURCE entry points reject null plans and
    arguments before touching the device."""
    L = chylib.lib()
    e = chylib.ChyExternal(1.0, 0.0, 0.0, 0.0, 0, 2)
    assert L.chy_plan_set_external(None, C.byref(e)) == 10
    assert L.chy_plan_set_external(None, None) == 10
    assert L.chy_plan_star_potential(None, None, 0, None) == 10
    a = chylib.ChySourceArgs()
    assert L.chy_source(None, C.byref(a), None) == 10
    assert L.chy_source(None, None, None) == 10
    assert C.sizeof(chylib.ChyDiag) == 8 + 8 + 4 + 4 + 64 + 16
    assert C.sizeof(chylib.ChyExternal) == 4 * 8 + 2 * 4
    assert C.sizeof(chylib.ChyBinary) == 2 * 8
    b = chylib.ChyBinary(1.0, 100.0)
    assert L.chy_plan_set_binary(None, C.byref(b)) == 10
    assert L.chy_source_binary(None, C.byref(a), C.byref(b), 1.0, None, None) == 10
    assert L.chy_source_binary(None, C.byref(a), None, 1.0, None, None) == 10
    assert C.sizeof(chylib.ChyTune) == 6 * 4 + 2 * 8 + 8
    # argument errors come with their own message
    o = chylib.ServerOpts()
    o.precision = 7
    srv = C.c_void_p()
    assert L.chy_server_create(C.byref(o), C.byref(srv)) == 10
    assert b"precision" in L.chy_last_error()
    t = chylib.ChyTune()
    assert L.chy_autotune_multi(0, None, None, None, None, 1, C.byref(t)) == 10
    assert L.chy_plan_set_schedule(None, C.byref(t)) == 10
    assert L.chy_plan_get_schedule(None, C.byref(t)) == 10
