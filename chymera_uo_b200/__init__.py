"""chymera_uo_b200 -- B200-native replacement of CHYMERA's gravitational
potential solve (SETBDY + BDYGEN + POT3, pot/boundary.f and pot/pot3.f).

The compute lives in ``libchy_pot3.so`` (CUDA, sm_100a) behind the C ABI in
``include/chy_pot3.h``; this module is a thin ctypes layer over it.  There is
no CPU fallback: if the library is missing, importing the solver fails.

Arrays use the reference's Fortran layout: RHO and PHI are
``(JMAX+2, KMAX+2, LMAX)`` float64 in column-major ("F") order.  Host arrays
(numpy) are staged through the device by the library; CUDA tensors (torch)
are used in place on the current stream.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libchy_pot3.so")

CHY_OK = 0
CHY_PREC_FP64 = 0
CHY_PREC_MIXED = 1
CHY_PREC_FP64_BLKTRI = 2
CHY_PTR_DEVICE = 0
CHY_PTR_HOST = 1
CHY_LITERAL_GCC = 0
CHY_LITERAL_R8 = 1
STAGES = ("forward+moments", "boundary integrals", "boundary potentials", "mode solves",
          "inverse+ghosts+zaxphi")


class ChyGrid(C.Structure):
    _fields_ = [("jmax", C.c_int), ("kmax", C.c_int), ("lmax", C.c_int),
                ("rof3n", C.c_double), ("zof3n", C.c_double),
                ("r", C.POINTER(C.c_double)), ("z", C.POINTER(C.c_double)),
                ("rhf", C.POINTER(C.c_double)), ("zhf", C.POINTER(C.c_double)),
                ("pi", C.c_double), ("grav", C.c_double),
                ("isym", C.c_int), ("maxtrm", C.c_int), ("redge", C.c_double),
                ("npoint", C.c_int), ("literal_kind", C.c_int)]


class ChyDiag(C.Structure):
    _fields_ = [("tmass", C.c_double), ("phichk", C.c_double), ("klocat", C.c_int),
                ("iterations", C.c_int), ("corr_rel", C.c_double * 8),
                ("indirectx", C.c_double), ("indirecty", C.c_double)]

    def as_dict(self):
        return {"tmass": self.tmass, "phichk": self.phichk, "klocat": self.klocat,
                "iterations": self.iterations,
                "corr_rel": list(self.corr_rel[: max(0, self.iterations)]),
                "indirectx": self.indirectx, "indirecty": self.indirecty}


class ChyExternal(C.Structure):
    """ExternalPot's inputs (pot/ExternalPot.f:1-80)."""
    _fields_ = [("mass_star", C.c_double), ("tmassacc", C.c_double),
                ("rpstar", C.c_double), ("phi_star", C.c_double),
                ("indirect", C.c_int), ("jmin", C.c_int)]


class ChyBinary(C.Structure):
    """The BINARY build's companion (pot/ExternalPot.f:57-69)."""
    _fields_ = [("mass_bin", C.c_double), ("a_bin", C.c_double)]


class ChySourceArgs(C.Structure):
    """SOURCE's arguments (radhydro/source.f:45-81); device pointers."""
    _fields_ = [("jmax", C.c_int), ("kmax", C.c_int), ("jmin", C.c_int), ("delt", C.c_double),
                ("rho", C.c_void_p), ("phi", C.c_void_p), ("omega", C.c_void_p), ("p", C.c_void_p),
                ("s", C.c_void_p), ("t", C.c_void_p), ("a", C.c_void_p)]


class ChyTune(C.Structure):
    _fields_ = [("streams", C.c_int), ("chunk", C.c_int), ("mode_ctas", C.c_int), ("blk_warps", C.c_int),
                ("blk_ctas_per_sm", C.c_int), ("mode_kernel", C.c_int), ("ms", C.c_double),
                ("ms_default", C.c_double), ("candidates", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget", C.c_longlong), ("precision", C.c_int), ("max_batch", C.c_int),
                ("arena_fraction", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_longlong), ("batches", C.c_longlong), ("size_classes", C.c_int),
                ("plan_bytes", C.c_longlong), ("arena_bytes", C.c_longlong)]


class ChyError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"chy status {status}: {msg}")
        self.status = status


_lib = None


def lib():
    """Loads libchy_pot3.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} missing: run `python -m chymera_uo_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, ip, i, d, ll = C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_double, C.c_longlong
        dpp = C.POINTER(C.c_void_p)
        L.chy_grid_defaults.argtypes = [C.POINTER(ChyGrid), i, i, i]
        L.chy_plan_create.argtypes = [C.POINTER(ChyGrid), i, i, C.POINTER(vp)]
        L.chy_plan_create.restype = i
        L.chy_plan_destroy.argtypes = [vp]
        L.chy_solve.argtypes = [vp, vp, vp, C.POINTER(ChyDiag), i, vp]
        L.chy_solve.restype = i
        L.chy_solve_batch.argtypes = [vp, i, dpp, dpp, C.POINTER(ChyDiag), i, vp]
        L.chy_solve_batch.restype = i
        L.chy_plan_set_coef.argtypes = [vp, vp]
        L.chy_plan_set_coef.restype = i
        L.chy_plan_set_refine.argtypes = [vp, i]
        L.chy_plan_set_refine.restype = i
        L.chy_plan_device_bytes.argtypes = [vp]
        L.chy_plan_device_bytes.restype = ll
        L.chy_plan_bytes_per_solve.argtypes = [vp]
        L.chy_plan_bytes_per_solve.restype = ll
        L.chy_status_string.argtypes = [i]
        L.chy_status_string.restype = C.c_char_p
        L.chy_last_error.restype = C.c_char_p
        L.chy_last_cuda_error.restype = i
        L.chy_plan_set_profiling.argtypes = [vp, i]
        L.chy_plan_set_profiling.restype = i
        L.chy_plan_stage_times.argtypes = [vp, C.POINTER(C.c_double), i, C.POINTER(ll)]
        L.chy_plan_stage_times.restype = i
        L.chy_plan_launch_count.argtypes = [vp]
        L.chy_plan_launch_count.restype = ll
        L.chy_dbg_fft.argtypes = [i, i, i, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.chy_dbg_fft.restype = i
        L.chy_dbg_realtr.argtypes = [i, i, i, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.chy_dbg_realtr.restype = i
        L.chy_dbg_table.argtypes = [C.POINTER(ChyGrid), C.c_char_p, C.POINTER(C.c_double), ll]
        L.chy_dbg_table.restype = ll
        L.chy_dbg_mixed_probe.argtypes = [vp, i]
        L.chy_dbg_mixed_probe.restype = i
        L.chy_dbg_mixed_kernel.argtypes = [vp]
        L.chy_dbg_mixed_kernel.restype = i
        L.chy_dbg_blktri.argtypes = [C.POINTER(ChyGrid), i, C.POINTER(C.c_double)]
        L.chy_dbg_blktri.restype = i
        L.chy_dbg_work.argtypes = [vp, C.c_char_p, C.POINTER(C.c_double), ll]
        L.chy_dbg_work.restype = ll
        L.chy_dbg_umma.argtypes = [vp, i, vp, vp, i]
        L.chy_dbg_umma.restype = i
        L.chy_solve_multi.argtypes = [i, dpp, dpp, dpp, vp]
        L.chy_solve_multi.restype = i
        L.chy_autotune_multi.argtypes = [i, dpp, dpp, dpp, vp, i, C.POINTER(ChyTune)]
        L.chy_autotune_multi.restype = i
        L.chy_plan_set_schedule.argtypes = [vp, C.POINTER(ChyTune)]
        L.chy_plan_set_schedule.restype = i
        L.chy_plan_get_schedule.argtypes = [vp, C.POINTER(ChyTune)]
        L.chy_plan_get_schedule.restype = i
        L.chy_solve_static.argtypes = [vp, vp, vp, vp]
        L.chy_solve_static.restype = i
        L.chy_plan_set_coef_host.argtypes = [vp, vp]
        L.chy_plan_set_coef_host.restype = i
        L.chy_server_create.argtypes = [C.POINTER(ServerOpts), C.POINTER(vp)]
        L.chy_server_create.restype = i
        L.chy_server_submit.argtypes = [vp, C.POINTER(ChyGrid), vp, vp, C.POINTER(ll)]
        L.chy_server_submit.restype = i
        L.chy_server_wait.argtypes = [vp, ll, C.POINTER(C.c_double)]
        L.chy_server_wait.restype = i
        L.chy_server_get_stats.argtypes = [vp, C.POINTER(ServerStats)]
        L.chy_server_get_stats.restype = i
        L.chy_server_destroy.argtypes = [vp]
        L.chy_plan_report.argtypes = [vp, C.c_char_p, ll]
        L.chy_plan_report.restype = ll
        L.chy_plan_set_binary.argtypes = [vp, C.POINTER(ChyBinary)]
        L.chy_plan_set_binary.restype = i
        L.chy_plan_set_external.argtypes = [vp, C.POINTER(ChyExternal)]
        L.chy_plan_set_external.restype = i
        L.chy_plan_star_potential.argtypes = [vp, vp, i, vp]
        L.chy_plan_star_potential.restype = i
        L.chy_source.argtypes = [vp, C.POINTER(ChySourceArgs), vp]
        L.chy_source.restype = i
        L.chy_source_binary.argtypes = [vp, C.POINTER(ChySourceArgs), C.POINTER(ChyBinary), C.c_double, vp, vp]
        L.chy_source_binary.restype = i
        _lib = L
    return _lib


def _check(status: int):
    if status != CHY_OK:
        L = lib()
        raise ChyError(status, f"{L.chy_status_string(status).decode()}: {L.chy_last_error().decode()}")


def grid(jmax: int, kmax: int, lmax: int, *, isym: int = 2, maxtrm: int = 10, redge: float = 0.0,
         npoint: int = 8, literal: str = "gcc", rof3n: float | None = None,
         zof3n: float | None = None, pi: float = 3.1415926535897932, grav: float = 1.0) -> ChyGrid:
    """A grid descriptor with the reference's defaults (radhydro/io.f:136-140,
    194-203; radhydro/3dhyd-main.f:166-167)."""
    g = ChyGrid()
    lib().chy_grid_defaults(C.byref(g), jmax, kmax, lmax)
    g.isym, g.maxtrm, g.redge, g.npoint = isym, maxtrm, redge, npoint
    g.literal_kind = CHY_LITERAL_R8 if literal == "r8" else CHY_LITERAL_GCC
    if rof3n is not None:
        g.rof3n = rof3n
    if zof3n is not None:
        g.zof3n = zof3n
    g.pi, g.grav = pi, grav
    return g


def _is_cuda_tensor(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


PRECISIONS = {"fp64": CHY_PREC_FP64, "mixed": CHY_PREC_MIXED, "blktri": CHY_PREC_FP64_BLKTRI}


def precision_code(precision: str) -> int:
    """CHY_PREC_* of a precision name: "blktri" (the reference's BLKTRI
    cyclic reduction in FP64, its rounding), "fp64" (FP64 eigenbasis solve)
    or "mixed" (tensor cores + FP64 refinement)."""
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}, not {precision!r}")
    return PRECISIONS[precision]


class Plan:
    """Per-grid tables + device work space for up to ``max_batch`` solves."""

    def __init__(self, g: ChyGrid, precision: str = "fp64", max_batch: int = 1):
        self.grid = g
        self.precision = precision
        self.shape = (g.jmax + 2, g.kmax + 2, g.lmax)
        p = C.c_void_p()
        prec = precision_code(precision)
        _check(lib().chy_plan_create(C.byref(g), prec, max_batch, C.byref(p)))
        self._p = p
        self.max_batch = max_batch

    def close(self):
        if getattr(self, "_p", None):
            lib().chy_plan_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        return lib().chy_plan_device_bytes(self._p)

    @property
    def bytes_per_solve(self) -> int:
        return lib().chy_plan_bytes_per_solve(self._p)

    @property
    def launches(self) -> int:
        return lib().chy_plan_launch_count(self._p)

    def set_refine(self, corrections: int):
        _check(lib().chy_plan_set_refine(self._p, corrections))

    def set_coef(self, coef_tensor):
        ptr = None if coef_tensor is None else coef_tensor.data_ptr()
        _check(lib().chy_plan_set_coef(self._p, ptr))

    def set_external(self, mass_star: float | None, tmassacc: float = 0.0, rpstar: float = 0.0,
                     phi_star: float = 0.0, indirect: bool = False, jmin: int = 2):
        """Adds the star potential of ExternalPot (pot/ExternalPot.f:1-80) to
        later solves; ``mass_star=None`` removes it."""
        if mass_star is None:
            _check(lib().chy_plan_set_external(self._p, None))
            return
        e = ChyExternal(mass_star, tmassacc, rpstar, phi_star, int(indirect), jmin)
        _check(lib().chy_plan_set_external(self._p, C.byref(e)))

    def report(self) -> str:
        """The IPRINT = 1 unit-3 text of the latest solve (chy_plan_report);
        needs the COEF output set (set_coef)."""
        n = lib().chy_plan_report(self._p, None, 0)
        if n < 0:
            _check(-n)
        buf = C.create_string_buffer(n + 1)
        lib().chy_plan_report(self._p, buf, n + 1)
        return buf.value.decode()

    def schedule(self) -> dict:
        """The plan's launch schedule (chy_plan_get_schedule)."""
        t = ChyTune()
        _check(lib().chy_plan_get_schedule(self._p, C.byref(t)))
        d = t.as_dict()
        for k in ("ms", "ms_default", "candidates"):
            d.pop(k)
        return d

    def set_schedule(self, streams: int = 0, chunk: int = 0, mode_ctas: int = 0, blk_warps: int = 8,
                     blk_ctas_per_sm: int = 2, mode_kernel: int = 0):
        """Sets the plan's launch schedule (chy_plan_set_schedule)."""
        t = ChyTune(streams, chunk, mode_ctas, blk_warps, blk_ctas_per_sm, mode_kernel, 0.0, 0.0, 0)
        _check(lib().chy_plan_set_schedule(self._p, C.byref(t)))

    def set_binary(self, mass_bin: float | None = 1.0, a_bin: float = 100.0):
        """Adds the BINARY build's companion term (pot/ExternalPot.f:57-69) to
        the external potential of later solves (MASSBIN = 1, ABIN = 100 in
        headers/units.h:25); ``mass_bin=None`` removes it."""
        if mass_bin is None:
            _check(lib().chy_plan_set_binary(self._p, None))
            return
        b = ChyBinary(mass_bin, a_bin)
        _check(lib().chy_plan_set_binary(self._p, C.byref(b)))

    def star_potential(self, out=None, stream=None):
        """STARPHI(JMAX+2, KMAX+2, LMAX) of the plan's external potential:
        into a CUDA tensor ``out`` (column-major), else a new numpy array."""
        if out is not None and _is_cuda_tensor(out):
            self._validate(out, True)
            _check(lib().chy_plan_star_potential(self._p, out.data_ptr(), CHY_PTR_DEVICE,
                                                 self._stream(stream)))
            return out
        if out is None:
            out = np.zeros(self.shape, dtype=np.float64, order="F")
        self._validate(out, False)
        _check(lib().chy_plan_star_potential(self._p, out.ctypes.data, CHY_PTR_HOST, stream or 0))
        return out

    def source(self, rho, phi, omega, p, s, t, a, delt: float, jmin: int = 2, stream=None, binary=None):
        """SOURCE's potential, pressure and rotation terms (radhydro/source.f:45-81)
        on CUDA tensors (column-major): s, t, a updated in place.  omega, p,
        s, t, a are (JMAX+2, KMAX+2, LMAX) of the hydro grid; rho, phi the
        plan's grid.

        binary: None (a BINARY = 0 build), or a dict with ``u`` (U, a hydro
        array), ``mass_star`` and optionally ``mass_bin`` (1) and ``a_bin``
        (100) for the BINARY build's terms (``chy_source_binary``)."""
        hshape = tuple(omega.shape)
        for x in (rho, phi):
            self._validate(x, True)
        hydro = (omega, p, s, t, a) + ((binary["u"],) if binary is not None else ())
        for x in hydro:
            if not _is_cuda_tensor(x) or tuple(x.shape) != hshape or str(x.dtype) != "torch.float64":
                raise ValueError(f"hydro arrays must be float64 CUDA tensors of one shape {hshape}")
            if x.stride() != (1, hshape[0], hshape[0] * hshape[1]):
                raise ValueError("device arrays must be column-major (Fortran) contiguous")
        if hshape[2] != self.shape[2]:
            raise ValueError("hydro and potential grids share LMAX")
        args = ChySourceArgs(hshape[0] - 2, hshape[1] - 2, jmin, delt, rho.data_ptr(), phi.data_ptr(),
                             omega.data_ptr(), p.data_ptr(), s.data_ptr(), t.data_ptr(), a.data_ptr())
        if binary is None:
            _check(lib().chy_source(self._p, C.byref(args), self._stream(stream)))
            return
        b = ChyBinary(float(binary.get("mass_bin", 1.0)), float(binary.get("a_bin", 100.0)))
        _check(lib().chy_source_binary(self._p, C.byref(args), C.byref(b), float(binary["mass_star"]),
                                       binary["u"].data_ptr(), self._stream(stream)))

    def set_profiling(self, on: bool):
        _check(lib().chy_plan_set_profiling(self._p, int(on)))

    def stage_times(self):
        ms = (C.c_double * 8)()
        calls = C.c_longlong(0)
        n = lib().chy_plan_stage_times(self._p, ms, 8, C.byref(calls))
        if n < 0:
            _check(-n)
        return {STAGES[i]: ms[i] for i in range(n)}, calls.value

    def debug_work(self, name: str, count: int) -> np.ndarray:
        """Copy of work array `name` of batch slot 0 (test hook)."""
        out = np.zeros(count)
        n = lib().chy_dbg_work(self._p, name.encode(), out.ctypes.data_as(C.POINTER(C.c_double)), count)
        if n < 0:
            _check(-n)
        return out[:n]

    def _stream(self, stream):
        if stream is not None:
            return stream
        import torch
        return torch.cuda.current_stream().cuda_stream

    def solve(self, rho, phi=None, diag: bool = False, stream=None):
        """SETBDY/BDYGEN/POT3 on one density.  numpy in -> numpy out (host
        staging); CUDA tensor in -> CUDA tensor out (in place if phi given)."""
        out = self.solve_batch([rho], None if phi is None else [phi], diag=diag, stream=stream)
        return out[0] if not diag else (out[0][0], out[1][0])

    def solve_batch(self, rhos, phis=None, diag: bool = False, stream=None):
        n = len(rhos)
        if n == 0:
            return ([], []) if diag else []
        dev = _is_cuda_tensor(rhos[0])
        if phis is None:
            if dev:
                import torch
                phis = [torch.zeros(self.shape[::-1], dtype=torch.float64, device=r.device).permute(2, 1, 0)
                        for r in rhos]
            else:
                phis = [np.zeros(self.shape, dtype=np.float64, order="F") for _ in rhos]
        for r, f in zip(rhos, phis):
            self._validate(r, dev)
            self._validate(f, dev)
        rp = (C.c_void_p * n)(*[self._ptr(r, dev) for r in rhos])
        fp = (C.c_void_p * n)(*[self._ptr(f, dev) for f in phis])
        d = (ChyDiag * n)() if diag else None
        st = self._stream(stream) if dev else (stream or 0)
        _check(lib().chy_solve_batch(self._p, n, rp, fp, d, CHY_PTR_DEVICE if dev else CHY_PTR_HOST,
                                     st))
        if diag:
            return phis, [d[i].as_dict() for i in range(n)]
        return phis

    def _validate(self, a, dev):
        if dev:
            if tuple(a.shape) != self.shape or a.dtype.__str__() != "torch.float64":
                raise ValueError(f"expected float64 tensor of shape {self.shape}")
            if a.stride() != (1, self.shape[0], self.shape[0] * self.shape[1]):
                raise ValueError("device arrays must be column-major (Fortran) contiguous")
        else:
            if a.shape != self.shape or a.dtype != np.float64 or not a.flags.f_contiguous:
                raise ValueError(f"expected Fortran-ordered float64 array of shape {self.shape}")

    @staticmethod
    def _ptr(a, dev):
        return a.data_ptr() if dev else a.ctypes.data


class Server:
    """Continuous-batching request loop (chy_server_*): submit host arrays
    (numpy, Fortran order; pinned memory gives full copy bandwidth) from any
    thread, wait for each ticket."""

    def __init__(self, precision: str = "mixed", hbm_budget: int = 0, max_batch: int = 8,
                 arena_fraction: float = 0.5):
        o = ServerOpts(hbm_budget, precision_code(precision), max_batch, arena_fraction)
        p = C.c_void_p()
        _check(lib().chy_server_create(C.byref(o), C.byref(p)))
        self._p = p
        self._keep = {}

    def submit(self, g: ChyGrid, rho: np.ndarray, phi: np.ndarray) -> int:
        shape = (g.jmax + 2, g.kmax + 2, g.lmax)
        for a in (rho, phi):
            if a.shape != shape or a.dtype != np.float64 or not a.flags.f_contiguous:
                raise ValueError(f"expected Fortran-ordered float64 array of shape {shape}")
        t = C.c_longlong(0)
        _check(lib().chy_server_submit(self._p, C.byref(g), rho.ctypes.data, phi.ctypes.data, C.byref(t)))
        self._keep[t.value] = (g, rho, phi)
        return t.value

    def wait(self, ticket: int) -> float:
        """Blocks until the request is done; returns its latency in ms."""
        ms = C.c_double(0.0)
        st = lib().chy_server_wait(self._p, ticket, C.byref(ms))
        self._keep.pop(ticket, None)
        _check(st)
        return ms.value

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().chy_server_get_stats(self._p, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self):
        if self._p:
            lib().chy_server_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pinned_fortran(shape):
    """A pinned host numpy array of the given Fortran shape (float64)."""
    import torch
    return torch.empty(tuple(shape[::-1]), dtype=torch.float64, pin_memory=True).numpy().transpose()


def solve_multi(plans, rhos, phis=None, stream=None):
    """Densities of several grids in one stream-ordered call (chy_solve_multi):
    rhos[i] (CUDA tensor, Fortran layout) is solved with plans[i]; returns the
    PHI tensors (new ones unless phis is given)."""
    import torch
    n = len(rhos)
    if len(plans) != n:
        raise ValueError("one plan per density")
    if phis is None:
        phis = [fortran_zeros_cuda(p.shape, device=r.device) for p, r in zip(plans, rhos)]
    for p, r, f in zip(plans, rhos, phis):
        p._validate(r, True)
        p._validate(f, True)
    pp = (C.c_void_p * n)(*[p._p.value for p in plans])
    rp = (C.c_void_p * n)(*[r.data_ptr() for r in rhos])
    fp = (C.c_void_p * n)(*[f.data_ptr() for f in phis])
    s = torch.cuda.current_stream() if stream is None else stream
    _check(lib().chy_solve_multi(n, pp, rp, fp, C.c_void_p(s.cuda_stream)))
    return phis


def autotune_multi(plans, rhos, phis=None, stream=None, repeats: int = 3) -> dict:
    """Picks the launch schedule of chy_solve_multi for this request set by
    timing candidates (chy_autotune_multi) and keeps it in the plans.
    Synchronises; call it before capturing a graph.  Returns the choice and
    the timings (ms per call, chosen and default)."""
    import torch
    n = len(rhos)
    if phis is None:
        phis = [fortran_zeros_cuda(p.shape, device=r.device) for p, r in zip(plans, rhos)]
    pp = (C.c_void_p * n)(*[p._p.value for p in plans])
    rp = (C.c_void_p * n)(*[r.data_ptr() for r in rhos])
    fp = (C.c_void_p * n)(*[f.data_ptr() for f in phis])
    s = torch.cuda.current_stream() if stream is None else stream
    t = ChyTune()
    _check(lib().chy_autotune_multi(n, pp, rp, fp, C.c_void_p(s.cuda_stream), repeats, C.byref(t)))
    return t.as_dict()


def fortran_zeros_cuda(shape, device="cuda"):
    """A column-major float64 CUDA tensor of the given Fortran shape."""
    import torch
    return torch.zeros(tuple(shape[::-1]), dtype=torch.float64, device=device).permute(
        *range(len(shape) - 1, -1, -1))


def to_cuda_fortran(a: np.ndarray, device="cuda"):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a.T)).to(device)
    return t.permute(*range(a.ndim - 1, -1, -1))
