"""chy_solve_static: the FP64 solve whose work space is a static device array
(no allocation during the call).  Collected last (file name) so it also runs
after every other GPU test; it passes alone in a fresh process as well.

Tolerance: the entry point runs the same kernels as chy_solve on the same
inputs, so the results must agree to rel. L2 <= 1e-15 (they are expected to
be bitwise equal)."""
import ctypes as C

import numpy as np
import pytest

from chymera_uo_b200 import synth

pytestmark = pytest.mark.gpu


def _rel(a, b):
    import torch
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def test_static_solve_matches_chy_solve_twice_in_a_row(chylib):
    import torch
    J, K, L = 64, 32, 64
    lib = chylib.lib()
    lib.chy_solve_static.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.chy_solve_static.restype = C.c_int
    plan = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    for seed in (5, 6):      # two calls in a row, different densities
        rho = chylib.to_cuda_fortran(synth.disk_density(J, K, L, seed, spiral=True, spectrum=True))
        ref = chylib.fortran_zeros_cuda(rho.shape)
        plan.solve(rho, ref)
        got = chylib.fortran_zeros_cuda(rho.shape)
        st = lib.chy_solve_static(plan._p, rho.data_ptr(), got.data_ptr(),
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert st == 0, lib.chy_last_error()
        torch.cuda.synchronize()
        assert _rel(got, ref) <= 1e-15
        assert torch.all(got[:, K + 1, :] == 0) and torch.all(got[J + 1, 0, :] == 0)


def test_static_solve_allocates_nothing(chylib):
    """The property the entry point exists for: after the first call on the
    device (which looks the static array up), two more calls leave the
    device's free memory and torch's allocator counters unchanged, and the
    plan's launch count grows by the kernels they ran."""
    import torch
    J, K, L = 64, 32, 64
    lib = chylib.lib()
    lib.chy_solve_static.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.chy_solve_static.restype = C.c_int
    plan = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    rho = chylib.to_cuda_fortran(synth.disk_density(J, K, L, 7, spiral=True, spectrum=True))
    outs = [chylib.fortran_zeros_cuda(rho.shape) for _ in range(3)]
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.chy_solve_static(plan._p, rho.data_ptr(), outs[0].data_ptr(), s) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    stats0 = torch.cuda.memory_stats()
    n0 = plan.launches
    for o in outs[1:]:
        assert lib.chy_solve_static(plan._p, rho.data_ptr(), o.data_ptr(), s) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    stats1 = torch.cuda.memory_stats()
    for key in ("allocation.all.allocated", "segment.all.allocated", "reserved_bytes.all.current"):
        assert stats1.get(key, 0) == stats0.get(key, 0), key
    assert plan.launches > n0
    assert torch.equal(outs[1], outs[0]) and torch.equal(outs[2], outs[0])


def test_static_solve_rejects_what_it_cannot_hold(chylib):
    import torch
    lib = chylib.lib()
    lib.chy_solve_static.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.chy_solve_static.restype = C.c_int
    big = chylib.Plan(chylib.grid(128, 64, 128), "fp64", 1)     # needs ~26 MiB of work space
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    assert lib.chy_solve_static(big._p, buf.data_ptr(), buf.data_ptr(), None) == 32   # CHY_ERR_CAPACITY
    assert b"static scratch holds 8388608 bytes" in lib.chy_last_error()
    mixed = chylib.Plan(chylib.grid(64, 32, 64), "mixed", 1)
    assert lib.chy_solve_static(mixed._p, buf.data_ptr(), buf.data_ptr(), None) == 12   # CHY_ERR_UNSUPPORTED
    assert lib.chy_solve_static(None, buf.data_ptr(), buf.data_ptr(), None) == 10       # CHY_ERR_ARG
