"""The mixed-precision path for grids the single-kernel mode solve does not
cover: JMAX > 256 (the 512 x 128 x 512 class of the serving workload) and
JMAX not a multiple of 16.  Five kernels per approximate solve (FP64
residual, tensor-core U product, FP32 radial sweeps, tensor-core V product,
FP64 update), the same refinement as the fused kernel.

Tolerance: rel. L2 <= 1e-10 over the write set against the oracle, as for
the fused mixed path."""
import functools

import numpy as np
import pytest

from chymera_uo_b200 import synth

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@functools.lru_cache(maxsize=None)
def oracle(J, K, L, seed):
    from oracle import oracle as O
    rho = synth.disk_density(J, K, L, seed, spiral=True, spectrum=True)
    o = O.Oracle(J, K, L, nthreads=8)
    return rho, np.array(o.solve(rho))


@pytest.mark.parametrize("J,K,L", [(512, 128, 512), (320, 64, 64), (72, 32, 64), (1024, 32, 64)])
def test_wide_grids_meet_1e10(chylib, J, K, L):
    rho, ref = oracle(J, K, L, 41)
    plan = chylib.Plan(chylib.grid(J, K, L), "mixed", 1)
    (phi,), (d,) = plan.solve_batch([rho], [np.zeros_like(rho, order="F")], diag=True)
    ws = (slice(0, J + 1), slice(0, K + 1))
    assert rel_l2(phi[ws], ref[ws]) < 1e-10
    assert d["iterations"] == 2 and d["corr_rel"][0] == pytest.approx(1.0) and d["corr_rel"][1] < 1e-4
    assert np.all(phi[:, K + 1, :] == 0.0) and np.all(phi[J + 1, 0, :] == 0.0)


def test_wide_refinement_converges(chylib):
    J, K, L = 512, 128, 512
    rho, ref = oracle(J, K, L, 41)
    ws = (slice(0, J + 1), slice(0, K + 1))
    errs = []
    for corrections in (0, 1, 2):
        plan = chylib.Plan(chylib.grid(J, K, L), "mixed", 1)
        plan.set_refine(corrections)
        phi = plan.solve(rho, np.zeros_like(rho, order="F"))
        errs.append(rel_l2(phi[ws], ref[ws]))
    assert errs[0] < 1e-4 and errs[1] < errs[0] * 1e-3 and errs[2] < 1e-11


def test_wide_batch_equals_single_solves_bitwise(chylib):
    import torch
    J, K, L = 320, 64, 64
    rhos = [chylib.to_cuda_fortran(synth.disk_density(J, K, L, 50 + s, spiral=True, spectrum=True))
            for s in range(3)]
    plan = chylib.Plan(chylib.grid(J, K, L), "mixed", 4)
    batch = plan.solve_batch(rhos)
    torch.cuda.synchronize()
    for r, b in zip(rhos, batch):
        single = plan.solve(r)
        torch.cuda.synchronize()
        assert torch.equal(single, b)
