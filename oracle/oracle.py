"""ctypes wrapper around the CPU oracle (oracle/pot3_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``.  The product library never loads it.

Parity status: unpinned against the reference binary (Fortran, no compiler
here, no reference fixtures).  See ``pot3_oracle.c`` for the restatement and
its documented deviations.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libpot3_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc -O2 -ffp-contract=off)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        vp, dp, ip, i, d = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int, C.c_double
        L.ora_new.restype = vp
        L.ora_new.argtypes = [i, i, i, i, i, i]
        L.ora_free.argtypes = [vp]
        for name in ("ora_phi", "ora_rho", "ora_r", "ora_z", "ora_rhf", "ora_zhf", "ora_coef",
                     "ora_massin", "ora_massout", "ora_rbdy", "ora_phac"):
            getattr(L, name).restype = dp
            getattr(L, name).argtypes = [vp]
        L.ora_jkmax.restype = i
        L.ora_jkmax.argtypes = [vp]
        L.ora_set_scalars.argtypes = [vp, d, d, d, d, d]
        L.ora_make_grid.argtypes = [vp, d, d]
        L.ora_setbdy.argtypes = [vp, i, i]
        L.ora_bdygen.restype = i
        L.ora_bdygen.argtypes = [vp, i, i, d]
        L.ora_pot3.argtypes = [vp, i, i]
        L.ora_inside.argtypes = [vp, dp]
        L.ora_fft.argtypes = [dp, dp, i, i, i, i, i]
        L.ora_realtr.argtypes = [dp, dp, i, i, i]
        L.ora_blktri_state_size.restype = i
        L.ora_blktri.argtypes = [vp, i, i, i, dp, dp, dp, i, i, dp, dp, dp, i, dp, ip, dp]
        L.ora_blktri_wsize.restype = i
        L.ora_external_pot.argtypes = [vp, d, d, d, d, i, i, dp, dp]
        L.ora_external_pot_binary.argtypes = [vp, d, d, d, d, i, i, i, d, d, dp, dp]
        L.ora_source.argtypes = [i, i, i, i, i, i, d, d, d, d, dp, dp, dp, dp, dp, dp, dp, dp]
        L.ora_source_binary.argtypes = [i, i, i, i, i, i, d, d, d, d, dp, dp, dp, dp, dp, dp, dp, dp, i, d, d, d,
                                        dp, dp]
        L.ora_blktri_wsize.argtypes = [i, i]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.c_contiguous or a.flags.f_contiguous)
    return a.ctypes.data_as(C.POINTER(C.c_double))


def fft(a: np.ndarray, b: np.ndarray, isn: int, literal_r8: bool, n: int | None = None) -> None:
    """In-place FFT(A,B,N,N,N,ISN) of pot/fft.f:73 on the first N entries."""
    if n is None:
        n = a.shape[0]
    lib().ora_fft(_dp(a), _dp(b), n, n, n, isn, int(literal_r8))


def realtr(a: np.ndarray, b: np.ndarray, n: int, isn: int, literal_r8: bool) -> None:
    """In-place REALTR(A,B,N,ISN) of pot/fft.f:2 (arrays of length >= N+1)."""
    lib().ora_realtr(_dp(a), _dp(b), n, isn, int(literal_r8))


def forward_real(x: np.ndarray, literal_r8: bool) -> np.ndarray:
    """POT3's forward transform of one column (pot/pot3.f:95-140): returns the
    LMAX mode coefficients in PHI order (cos 0..N, then sin 1..N-1), scaled by
    SF1 = 0.5/N."""
    L = x.shape[0]
    n = L // 2
    a = np.zeros(L + 2)
    b = np.zeros(L + 2)
    a[:n] = x[0::2]
    b[:n] = x[1::2]
    fft(a, b, 1, literal_r8, n)
    realtr(a, b, n, 1, literal_r8)
    sf1 = 0.5 / n if literal_r8 else float(np.float32(0.5) / np.float32(n))
    out = np.empty(L)
    out[: n + 1] = a[: n + 1] * sf1
    out[n + 1:] = b[1:n] * sf1
    return out


def inverse_real(modes: np.ndarray, literal_r8: bool) -> np.ndarray:
    """POT3's inverse transform of one column (pot/pot3.f:260-279)."""
    L = modes.shape[0]
    n = L // 2
    a = np.zeros(L + 2)
    b = np.zeros(L + 2)
    a[: n + 1] = modes[: n + 1]
    b[1:n] = modes[n + 1:]
    realtr(a, b, n, -1, literal_r8)
    fft(a, b, -1, literal_r8, n)
    x = np.empty(L)
    x[0::2] = 0.5 * a[:n]
    x[1::2] = 0.5 * b[:n]
    return x


class Oracle:
    """One reference-shaped context: COMMON blocks sized for (JMAX, KMAX, LMAX)."""

    def __init__(self, jmax: int, kmax: int, lmax: int, literal_r8: bool = False,
                 nthreads: int = 1, want_coef: bool = False):
        self.J, self.K, self.L = jmax, kmax, lmax
        self.literal_r8 = literal_r8
        self._c = lib().ora_new(jmax, kmax, lmax, int(literal_r8), nthreads, int(want_coef))
        shape = (jmax + 2, kmax + 2, lmax)
        cnt = shape[0] * shape[1] * shape[2]
        as_arr = np.ctypeslib.as_array
        self.phi = as_arr(lib().ora_phi(self._c), (cnt,)).reshape(shape, order="F")
        self.rho = as_arr(lib().ora_rho(self._c), (cnt,)).reshape(shape, order="F")
        self.r = as_arr(lib().ora_r(self._c), (jmax + 2,))
        self.z = as_arr(lib().ora_z(self._c), (kmax + 2,))
        self.rhf = as_arr(lib().ora_rhf(self._c), (jmax + 2,))
        self.zhf = as_arr(lib().ora_zhf(self._c), (kmax + 2,))
        self.coef = None
        if want_coef:
            cs = (jmax + 2, kmax + 2, lmax // 2, 2)
            self.coef = as_arr(lib().ora_coef(self._c), (int(np.prod(cs)),)).reshape(cs, order="F")
        jkm1 = 2 * jmax + kmax - 1
        self.massin = as_arr(lib().ora_massin(self._c), (2 * 66 * jkm1,)).reshape((2, 66, jkm1), order="F")
        self.massout = as_arr(lib().ora_massout(self._c), (2 * 66 * jkm1,)).reshape((2, 66, jkm1), order="F")
        self.rbdy = as_arr(lib().ora_rbdy(self._c), (jkm1,))
        self.phac = as_arr(lib().ora_phac(self._c), (kmax + 2,))

    def close(self):
        if self._c:
            lib().ora_free(self._c)
            self._c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_grid(self, delr: float, delz: float, pi: float = 3.1415926535897932,
                 grav: float = 1.0):
        """radhydro/io.f:136-140,194-203: PI, GRAV, DTHETA=2*PI/LMAX, R/Z/RHF/ZHF."""
        lib().ora_make_grid(self._c, delr, delz)
        dtheta = 2.0 * pi / float(self.L)
        lib().ora_set_scalars(self._c, delr, delz, dtheta, pi, grav)

    def setbdy(self, ncall: int = 0, isym: int = 2):
        lib().ora_setbdy(self._c, ncall, isym)

    def bdygen(self, maxtrm: int = 10, isym: int = 2, redge: float = 0.0) -> int:
        return lib().ora_bdygen(self._c, maxtrm, isym, redge)

    def pot3(self, npoint: int = 8, iprint: int = 0):
        lib().ora_pot3(self._c, npoint, iprint)

    def inside(self):
        out = np.zeros(3)
        lib().ora_inside(self._c, _dp(out))
        return {"tmass": out[0], "phichk": out[1], "klocat": int(out[2])}

    def external_pot(self, mass_star: float, tmassacc: float = 0.0, rpstar: float = 0.0,
                     phi_star: float = 0.0, indirect: bool = False, jmin: int = 2,
                     binary: bool = False, mass_bin: float = 1.0, a_bin: float = 100.0):
        """ExternalPot (pot/ExternalPot.f:1-80) on the context's PHI: adds
        STARPHI in place, and with `binary` the BINARY build's companion term.
        Returns (STARPHI, (INDIRECTX, INDIRECTY))."""
        sp = np.zeros((self.J + 2, self.K + 2, self.L), order="F")
        ixy = np.zeros(2)
        lib().ora_external_pot_binary(self._c, mass_star, tmassacc, rpstar, phi_star, int(indirect), jmin,
                                      int(binary), mass_bin, a_bin, _dp(sp), _dp(ixy))
        return sp, (float(ixy[0]), float(ixy[1]))

    def solve(self, rho: np.ndarray, delr: float | None = None, delz: float | None = None,
              isym: int = 2, maxtrm: int = 10, redge: float = 0.0, npoint: int = 8,
              phi_init: np.ndarray | None = None) -> np.ndarray:
        """SETBDY(0) + BDYGEN + POT3 as radhydro/io.f:212-218 calls them.
        Returns a copy of PHI (Fortran order)."""
        if delr is None:
            delr = 1.0 / self.J
        if delz is None:
            delz = 0.5 / self.K
        self.set_grid(delr, delz)
        self.rho[...] = rho
        if phi_init is None:
            self.phi[...] = 0.0
        else:
            self.phi[...] = phi_init
        self.setbdy(0, isym)
        rc = self.bdygen(maxtrm, isym, redge)
        if rc != 0:
            raise RuntimeError("BDYGEN called before SETBDY")
        self.pot3(npoint, 0)
        return np.array(self.phi, order="F", copy=True)


def source(r, rho, phi, omega, p, s, t, a, delt, dr, dz, dtheta, jmin=2, binary=None):
    """SOURCE's first loop nest (radhydro/source.f:45-81) on Fortran-ordered
    arrays: omega, p, s, t, a of the hydro grid (JMAX+2, KMAX+2, LMAX); rho,
    phi of the potential grid.  s, t, a are updated in place.

    binary: None for a BINARY = 0 build, else a dict with mass_star, mass_bin,
    a_bin, rhf (RHF of the potential grid) and u (U, hydro grid) for the
    BINARY build's terms (source.f:38-40, 61-62, 76-77)."""
    j2, k2, lmax = omega.shape
    j2p, k2p, _ = rho.shape
    for x in (rho, phi, omega, p, s, t, a):
        assert x.dtype == np.float64 and x.flags.f_contiguous
    for x in (omega, p, s, t, a):
        assert x.shape == (j2, k2, lmax)
    assert phi.shape == rho.shape and r.shape[0] >= j2p
    args = (j2 - 2, k2 - 2, lmax, j2p, k2p, jmin, delt, dr, dz, dtheta, _dp(np.ascontiguousarray(r)),
            _dp(rho), _dp(phi), _dp(omega), _dp(p), _dp(s), _dp(t), _dp(a))
    if binary is None:
        lib().ora_source(*args)
        return
    u = binary["u"]
    rhf = np.ascontiguousarray(binary["rhf"], dtype=np.float64)
    assert u.dtype == np.float64 and u.flags.f_contiguous and u.shape == (j2, k2, lmax)
    assert rhf.shape[0] >= j2p
    lib().ora_source_binary(*args, 1, float(binary["mass_star"]), float(binary["mass_bin"]), float(binary["a_bin"]),
                            _dp(rhf), _dp(u))


def blktri_solve(an, bn, cn, am, bm, cm, y):
    """BLKTRI(0,...) then BLKTRI(1,...) on one system with NP=MP=1 as POT3
    calls it (pot/pot3.f:234-239).  y has shape (M, N) and is solved in place
    (returned).  Returns (y, ierror)."""
    n = an.shape[0]
    m = am.shape[0]
    w = np.zeros(lib().ora_blktri_wsize(m + 1, n + 1) + 4 * n + 64)
    state = C.create_string_buffer(max(256, lib().ora_blktri_state_size()))
    ierr = C.c_int(0)
    yf = np.asfortranarray(y, dtype=np.float64)
    args = [C.cast(state, C.c_void_p)]
    for iflg in (0, 1):
        lib().ora_blktri(args[0], iflg, 1, n, _dp(an), _dp(bn), _dp(cn), 1, m, _dp(am), _dp(bm),
                         _dp(cm), m, _dp(yf), C.byref(ierr), _dp(w))
        if iflg == 0 and ierr.value != 0:
            return yf, ierr.value
    return yf, ierr.value


def blktri_roots(an, bn, cn, m):
    """The work array of BLKTRI(IFLG=0) (NP=MP=1): COMPB's root table B
    followed by the shifted CN copy (pot/blktri.f:35-46)."""
    n = an.shape[0]
    w = np.zeros(lib().ora_blktri_wsize(m + 1, n + 1) + 4 * n + 64)
    state = C.create_string_buffer(max(256, lib().ora_blktri_state_size()))
    ierr = C.c_int(0)
    y = np.zeros((m, n), order="F")
    am = np.zeros(m)
    lib().ora_blktri(C.cast(state, C.c_void_p), 0, 1, n, _dp(an), _dp(bn), _dp(cn), 1, m, _dp(am), _dp(am),
                     _dp(am), m, _dp(y), C.byref(ierr), _dp(w))
    return w, ierr.value
