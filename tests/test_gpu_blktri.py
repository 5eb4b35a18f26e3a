"""The BLKTRI-order FP64 path (CHY_PREC_FP64_BLKTRI) on the GPU.

Its mode solve replays the reference's BLKTRI (pot/blktri.f) with the
reference's operations in the reference's order, so:
  * the solved modes equal the host replay of the recorded schedule (itself
    bit-identical to the oracle's BLKTRI, tests/test_host_blktri.py) bit for
    bit;
  * PHI matches the oracle's POT3 to <= 1e-12 relative L2 over the write set
    at every size, 256x128x256 included (the only differences left are the
    boundary sums' fixed summation order, ~1e-15).
"""
import ctypes as C
import functools

import numpy as np
import pytest

from chymera_uo_b200 import synth

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def write_set(J, K):
    return (slice(0, J + 1), slice(0, K + 1), slice(None))


@functools.lru_cache(maxsize=None)
def oracle_result(cfg, literal="gcc", seed=None):
    from oracle import oracle as O
    if seed is None:
        rho, g = synth.config_density(cfg)
    else:
        J, K, L = cfg
        rho, g = synth.disk_density(J, K, L, seed, spiral=True, spectrum=True), synth.default_grid(J, K, L)
    o = O.Oracle(g.jmax, g.kmax, g.lmax, literal_r8=(literal == "r8"), nthreads=8)
    phi = o.solve(rho)
    return rho, phi, o.inside()


def solve(chy, rho, J, K, L, nb=1, **gkw):
    plan = chy.Plan(chy.grid(J, K, L, **gkw), "blktri", nb)
    (out,), (d,) = plan.solve_batch([rho], [np.zeros_like(rho, order="F")], diag=True)
    return out, d, plan


def test_large_grid_meets_1e12(chylib):
    """The plain FP64 pot3 at 256x128x256 (seeded disk with an m=2 spiral)
    against the oracle: <= 1e-12 relative L2 over the write set."""
    rho, ref, dref = oracle_result(2)
    phi, d, _ = solve(chylib, rho, 256, 128, 256)
    ws = write_set(256, 128)
    assert rel_l2(phi[ws], ref[ws]) < 1e-12
    assert abs(d["tmass"] - dref["tmass"]) <= 1e-13 * dref["tmass"]
    assert d["klocat"] == dref["klocat"]


@pytest.mark.parametrize("literal", ["gcc", "r8"])
def test_small_grid_meets_1e12(chylib, literal):
    rho, ref, dref = oracle_result(1, literal)
    phi, d, _ = solve(chylib, rho, 64, 32, 64, literal=literal)
    ws = write_set(64, 32)
    assert rel_l2(phi[ws], ref[ws]) < 1e-12
    assert abs(d["phichk"] - dref["phichk"]) <= 1e-6 * abs(dref["phichk"])


@pytest.mark.parametrize("J,K,L", [(128, 64, 128), (64, 32, 256), (80, 32, 64), (65, 32, 64), (256, 64, 64),
                                   (32, 8, 32), (512, 128, 512)])
def test_other_grid_sizes(chylib, J, K, L):
    rho, ref, _ = oracle_result((J, K, L), seed=31)
    phi, _, _ = solve(chylib, rho, J, K, L)
    ws = write_set(J, K)
    assert rel_l2(phi[ws], ref[ws]) < 1e-12


def test_modes_equal_host_replay_bitwise(chylib, ora):
    """The device's solved modes equal the recorded schedule replayed on the
    host, bit for bit, for every mode.  The right-hand side is rebuilt from
    the oracle's forward transform (which the device transform equals bit for
    bit) and the device's boundary rows, with POT3's folds in POT3's order."""
    J, K, L = 64, 32, 64
    M, NZ = J - 1, K - 1
    rho = synth.disk_density(J, K, L, 5, spiral=True, spectrum=True)
    g = chylib.grid(J, K, L)
    plan = chylib.Plan(g, "blktri", 1)
    plan.solve_batch([rho])
    X = plan.debug_work("X", L * K * J).reshape(L, K, J)
    F = np.zeros((L, NZ, M))
    for k in range(NZ):
        for j in range(M):
            F[:, k, j] = ora.forward_real(rho[j + 1, k + 1, :].copy(), False)
    sc = np.zeros(8)
    assert chylib.lib().chy_dbg_table(C.byref(g), b"scalars", sc.ctypes.data_as(C.POINTER(C.c_double)), 8) == 8
    pig4, cmmax, cnmax = sc[1], sc[2], sc[4]
    for l in range(L):
        y = np.asfortranarray((pig4 * F[l]).T)            # Y(j, k)
        y[:, NZ - 1] = y[:, NZ - 1] - cnmax * X[l, NZ, :M]
        y[M - 1, :] = y[M - 1, :] - cmmax * X[l, :NZ, M]
        assert chylib.lib().chy_dbg_blktri(C.byref(g), l, y.ctypes.data_as(C.POINTER(C.c_double))) == 0
        assert np.array_equal(y, X[l, :NZ, :M].T), l


def test_batch_and_host_paths_equal_single_device_solves(chylib):
    """A batch (several groups of 32 modes per solve) equals single solves
    bit for bit, through device and host pointers."""
    import torch
    J, K, L = 64, 32, 64
    rhos = [synth.disk_density(J, K, L, 60 + s, spiral=True, spectrum=True) for s in range(5)]
    plan = chylib.Plan(chylib.grid(J, K, L), "blktri", 4)
    rd = [chylib.to_cuda_fortran(r) for r in rhos]
    batch = plan.solve_batch(rd)
    torch.cuda.synchronize()
    host = plan.solve_batch(rhos, [np.zeros_like(r, order="F") for r in rhos])
    for r, b, h in zip(rd, batch, host):
        single = plan.solve(r)
        torch.cuda.synchronize()
        assert torch.equal(single, b)
        assert np.array_equal(h, b.cpu().numpy())


def test_write_set_untouched_cells(chylib):
    rho, _, _ = oracle_result(1)
    J, K = 64, 32
    plan = chylib.Plan(chylib.grid(J, K, 64), "blktri", 1)
    phi = plan.solve(rho, np.full_like(rho, 7.0, order="F"))
    assert np.all(phi[:, K + 1, :] == 7.0) and np.all(phi[J + 1, 0, :] == 7.0)
    assert np.all(np.isfinite(phi))


@pytest.mark.parametrize("nw,cps", [(4, 2), (4, 4), (8, 1), (16, 1)])
def test_stage_schedules_give_the_same_modes(chylib, nw, cps):
    """The stage schedule (warps per CTA, CTAs per SM) only changes which warp
    runs which task: PHI is bitwise the default schedule's."""
    import torch
    J, K, L = 64, 32, 64
    rho = chylib.to_cuda_fortran(synth.disk_density(J, K, L, 11, spiral=True, spectrum=True))
    plan = chylib.Plan(chylib.grid(J, K, L), "blktri", 2)
    ref = plan.solve_batch([rho, rho])
    plan.set_schedule(blk_warps=nw, blk_ctas_per_sm=cps)
    assert plan.schedule()["blk_warps"] == nw
    got = plan.solve_batch([rho, rho])
    torch.cuda.synchronize()
    assert torch.equal(got[0], ref[0]) and torch.equal(got[1], ref[0])


@functools.lru_cache(maxsize=None)
def oracle_variant(isym, maxtrm, npoint, redge):
    from oracle import oracle as O
    rho, g = synth.config_density(1)
    o = O.Oracle(64, 32, 64, nthreads=8)
    phi = o.solve(rho, isym=isym, maxtrm=maxtrm, redge=redge, npoint=npoint)
    return rho, phi


@pytest.mark.parametrize("isym,maxtrm,npoint,redge", [(1, 10, 8, 0.0), (3, 8, 8, 0.0), (2, 4, 7, 0.0),
                                                      (-2, 10, 8, 0.0), (2, 10, 8, 0.6)])
def test_call_parameter_variants(chylib, isym, maxtrm, npoint, redge):
    """ISYM, MAXTRM, NPOINT and REDGE as BDYGEN/ZAXPHI take them
    (pot/boundary.f:97-105, pot/pot3.f:328-348), through the BLKTRI-order
    mode solve: within 1e-12 of the oracle."""
    rho, ref = oracle_variant(isym, maxtrm, npoint, redge)
    phi, _, _ = solve(chylib, rho, 64, 32, 64, isym=isym, maxtrm=maxtrm, npoint=npoint, redge=redge)
    ws = write_set(64, 32)
    assert rel_l2(phi[ws], ref[ws]) < 1e-12
