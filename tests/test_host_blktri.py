"""The BLKTRI-order FP64 mode solve's host side, checked without a GPU.

The library records the reference's BLKTRI (pot/blktri.f) once per grid:
COMPB's root table and every PRDCT call of BLKTR1 as a program of
tridiagonal passes and right-hand-side updates, grouped into stages of
independent tasks.  The device kernel replays exactly those operations.
Here the same replay runs on the host (chy_dbg_blktri) and must equal the
oracle's line-by-line BLKTRI bit for bit, for every kind of mode.
"""
import ctypes as C

import numpy as np
import pytest


def dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def table(chy, g, name, n):
    out = np.zeros(n)
    m = chy.lib().chy_dbg_table(C.byref(g), name.encode(), dp(out), n)
    assert m >= 0, (name, m)
    return out[:m]


def stretched_grid(chy, J, K, L):
    """A grid whose vertical spacing grows with height, so that every
    sub-block of the vertical operator (and so every COMPB root set) differs."""
    g = chy.grid(J, K, L)
    dz = 0.5 / K
    zhf = np.array([(k - 1.5) * dz * (1.0 + 0.3 * (k / K) ** 2) for k in range(1, K + 3)])
    z = np.concatenate([[zhf[0] - 0.5 * dz], 0.5 * (zhf[:-1] + zhf[1:])])
    keep = (np.ascontiguousarray(z), np.ascontiguousarray(zhf))
    g.z = keep[0].ctypes.data_as(C.POINTER(C.c_double))
    g.zhf = keep[1].ctypes.data_as(C.POINTER(C.c_double))
    return g, keep


GRIDS = [(16, 8, 32), (64, 32, 64), (128, 64, 128), (256, 128, 256), (512, 128, 512)]


@pytest.mark.parametrize("J,K,L", GRIDS + [("stretched", 32, 64)])
def test_roots_equal_oracle_compb(chylib, ora, J, K, L):
    """COMPB's root table B and the shifted CN copy (pot/blktri.f:35-46,
    264-344) equal the oracle's BLKTRI(IFLG=0) work array bit for bit."""
    keep = None
    if J == "stretched":
        J = 64
        g, keep = stretched_grid(chylib, J, K, L)
    else:
        g = chylib.grid(J, K, L)
    NZ, M = K - 1, J - 1
    an, bn, cn = table(chylib, g, "an", NZ), table(chylib, g, "bn", NZ), table(chylib, g, "cn", NZ)
    roots = table(chylib, g, "blk_roots", 1 << 16)
    cns = table(chylib, g, "blk_cns", NZ)
    w, ierr = ora.blktri_roots(an, bn, cn, M)
    assert ierr == 0
    nr = roots.size
    assert np.array_equal(roots, w[:nr])
    assert np.array_equal(cns, w[nr:nr + NZ])


@pytest.mark.parametrize("J,K,L", GRIDS + [("stretched", 32, 64)])
def test_replay_equals_oracle_blktri(chylib, ora, J, K, L):
    """The recorded schedule replayed on the host solves every kind of mode
    (m = 0, odd and even m, the Nyquist cosine, sine modes) bit for bit as
    the oracle's BLKTRI does, on random right-hand sides."""
    keep = None
    if J == "stretched":
        J = 64
        g, keep = stretched_grid(chylib, J, K, L)
    else:
        g = chylib.grid(J, K, L)
    NZ, M, N = K - 1, J - 1, L // 2
    an, bn, cn = table(chylib, g, "an", NZ), table(chylib, g, "bn", NZ), table(chylib, g, "cn", NZ)
    am, cm = table(chylib, g, "am", M), table(chylib, g, "cm", M)
    bm_all = table(chylib, g, "blk_bm", L * M).reshape(L, M)
    rng = np.random.default_rng(J + K + L)
    modes = sorted({0, 1, 2, 3, N - 1, N, N + 1, L - 1})
    for l in modes:
        y = np.asfortranarray(rng.standard_normal((M, NZ)))
        ref, ierr = ora.blktri_solve(an, bn, cn, am, bm_all[l], cm, y.copy(order="F"))
        assert ierr == 0
        got = y.copy(order="F")
        assert chylib.lib().chy_dbg_blktri(C.byref(g), l, dp(got)) == 0
        assert np.array_equal(got, ref), (l, float(np.abs(got - ref).max()))


@pytest.mark.parametrize("J,K,L", [(64, 32, 64), (256, 128, 256), (16, 8, 32)])
def test_bm_is_pot3s_expression(chylib, J, K, L):
    """BM of each mode (pot/pot3.f:226-230) restated in numpy with POT3's
    order of operations; the kernel's lane-interleaved table holds the same
    values with lane -> mode (32 * block + lane) mod L."""
    g = chylib.grid(J, K, L)
    M, N = J - 1, L // 2
    am, cm, cc = table(chylib, g, "am", M), table(chylib, g, "cm", M), table(chylib, g, "cc", M)
    xlamm = table(chylib, g, "xlamm", N + 1)
    sc = table(chylib, g, "scalars", 8)
    cmmax, ammin = sc[2], sc[3]
    bm_all = table(chylib, g, "blk_bm", L * M).reshape(L, M)
    for l in range(L):
        m = l if l <= N else l - N
        powrm = 1.0 if m % 2 == 0 else -1.0
        x2 = 2.0 * (xlamm[m] - 1.0)
        ref = np.empty(M)
        ref[0] = (-cm[0] + (powrm - 1.0) * ammin) + x2 * cc[0]
        for j in range(1, M - 1):
            ref[j] = (-cm[j] - am[j]) + x2 * cc[j]
        ref[M - 1] = (-cmmax - am[M - 1]) + x2 * cc[M - 1]
        assert np.array_equal(bm_all[l], ref), l
    nblk = max(1, L // 32)
    tab = table(chylib, g, "blk_bm_table", nblk * M * 32).reshape(nblk, M, 32)
    for b in range(nblk):
        for lane in range(32):
            assert np.array_equal(tab[b, :, lane], bm_all[(32 * b + lane) % L])
