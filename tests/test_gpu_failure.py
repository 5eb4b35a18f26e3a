"""Failure reporting of the mixed path's bounded waits, without a GPU fault.

Every wait of the tensor-core mode solve on a copy or a product is bounded;
when one runs out the CTA stops, drains what it has in flight, writes NaN
into the modes it left unsolved, sets the plan's device error word and
exits.  The test hook chy_dbg_mixed_probe makes every CTA first wait on a
barrier that nothing arrives on -- before any copy or product is issued --
so the wait runs out on purpose and the whole failure path runs with
nothing in flight.
"""
import numpy as np
import pytest

from chymera_uo_b200 import synth

pytestmark = pytest.mark.gpu

J, K, L = 64, 32, 64
TIMEOUT = 31   # CHY_ERR_TIMEOUT


def interior(a):
    return a[1:J, 1:K, :]


@pytest.mark.parametrize("mode_kernel", [1, 2])
def test_expired_wait_is_reported_and_the_next_solve_is_clean(chylib, mode_kernel):
    """Both fused mode-solve kernels: k_mode_mixed (1) and the CTA pairs of
    k_mode_pair (2), whose CTAs also end with a cluster barrier."""
    import torch
    rho = synth.disk_density(J, K, L, 9, spiral=True, spectrum=True)
    plan = chylib.Plan(chylib.grid(J, K, L), "mixed", 2)
    plan.set_schedule(mode_kernel=mode_kernel)
    lib = chylib.lib()
    ref = plan.solve(rho, np.zeros_like(rho, order="F"))
    assert np.all(np.isfinite(ref))
    try:
        assert lib.chy_dbg_mixed_probe(plan._p, 1000) == 0
        # host pointers: the call synchronises and returns the status; the
        # unsolved modes reach PHI as NaN
        phi = np.zeros_like(rho, order="F")
        with pytest.raises(chylib.ChyError) as e:
            plan.solve(rho, phi)
        assert e.value.status == TIMEOUT
        assert np.isnan(interior(phi)).all()
        # device pointers with diagnostics: the same call reports it
        rd = chylib.to_cuda_fortran(rho)
        with pytest.raises(chylib.ChyError) as e:
            plan.solve(rd, diag=True)
        assert e.value.status == TIMEOUT
        # device pointers without diagnostics: asynchronous, PHI carries NaN and
        # the plan's next synchronising call reports the expiry
        pd = plan.solve(rd)
        torch.cuda.synchronize()
        assert torch.isnan(pd[1:J, 1:K, :]).all()
        assert lib.chy_dbg_mixed_probe(plan._p, 0) == 0
        with pytest.raises(chylib.ChyError) as e:
            plan.solve(rho, np.zeros_like(rho, order="F"))
        assert e.value.status == TIMEOUT
    finally:
        lib.chy_dbg_mixed_probe(plan._p, 0)
    # nothing is left over: the next solves are clean and equal the first
    again = plan.solve(rho, np.zeros_like(rho, order="F"))
    assert np.array_equal(again, ref)
    out, d = plan.solve(chylib.to_cuda_fortran(rho), diag=True)
    assert np.array_equal(out.cpu().numpy(), ref) and d["iterations"] == 2


def test_probe_needs_a_mixed_plan(chylib):
    plan = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    assert chylib.lib().chy_dbg_mixed_probe(plan._p, 10) == 10
