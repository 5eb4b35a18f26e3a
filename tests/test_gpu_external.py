"""ExternalPot (pot/ExternalPot.f:1-80) fused into the inverse transform, on
the GPU through the C ABI, against the oracle's restatement.

STARPHI depends only on the grid and the star position, and the library
evaluates it in the reference's order of operations with every product and
sum rounded on its own, so:
  * STARPHI from chy_plan_star_potential equals the oracle's bit for bit;
  * PHI with the external potential equals (PHI without it) + STARPHI bit
    for bit, in every cell, for both precisions and both pointer kinds.
The INDIRECT star position sums the disk's mass moment in a different order
than the reference's serial loop.  Its terms cancel (the moment of a nearly
axisymmetric disk is small), so the bar is on the scale of the terms: 1e-12
of their absolute sum, below the serial loop's own worst-case rounding
(n * 2**-53 of it, 1.5e-11 at 64x32x64).  The whole chain against the
oracle's POT3 + ExternalPot: the FP64 path's 1e-12 relative L2.
"""
import math

import numpy as np
import pytest

from chymera_uo_b200 import synth

pytestmark = pytest.mark.gpu

J, K, L = 64, 32, 64
STAR = dict(mass_star=1.0, tmassacc=0.0125, rpstar=0.0031, phi_star=0.7)


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def density(seed=1):
    return synth.disk_density(J, K, L, seed, spiral=True, spectrum=True)


def phi_start(seed=7):
    # nonzero everywhere, so the cells POT3 leaves alone show whether they
    # were carried through and updated
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal((J + 2, K + 2, L)))


def oracle_chain(rho, phi0, **star):
    from oracle import oracle as O
    o = O.Oracle(J, K, L, nthreads=8)
    o.solve(rho, phi_init=phi0)
    sp, ixy = o.external_pot(**star)
    return np.array(o.phi, order="F"), sp, ixy


def moment_scale(rho, jmin, mass_star):
    """Absolute sum of the INDIRECT moment's terms over MASS_STAR."""
    rhf = (np.arange(1, J + 3) - 2 + 0.5) / J
    dth = 2.0 * 3.1415926535897932 / L
    r = rhf[jmin - 1:J + 1, None, None]
    return float(np.sum(np.abs(rho[jmin - 1:J + 1, 1:K + 1, :] * r * r)) * (1.0 / J) * (0.5 / K) * 2 * dth) / mass_star


def check_shift(d, ix, iy, rho, jmin, mass_star):
    tol = 1e-12 * moment_scale(rho, jmin, mass_star)
    assert abs(d["indirectx"] - ix) <= tol
    assert abs(d["indirecty"] - iy) <= tol


def host_solve(chy, plan, rho, phi0, diag=True):
    phi = phi0.copy(order="F")
    (out,), (d,) = plan.solve_batch([rho], [phi], diag=True)
    return out, d


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_add_is_bitwise_v_plus_starphi(chylib, precision):
    rho, phi0 = density(), phi_start()
    plan = chylib.Plan(chylib.grid(J, K, L), precision, 1)
    v, _ = host_solve(chylib, plan, rho, phi0)
    plan.set_external(**STAR)
    e, d = host_solve(chylib, plan, rho, phi0)
    _, sp_ref, (ix, iy) = oracle_chain(rho, phi0, **STAR)
    sp = plan.star_potential()
    assert np.array_equal(sp, sp_ref)
    assert np.array_equal(e, v + sp_ref)
    # the cells POT3 never writes: the caller's values plus STARPHI
    assert np.array_equal(e[:, K + 1, :], phi0[:, K + 1, :] + sp_ref[:, K + 1, :])
    assert np.array_equal(e[J + 1, 0, :], phi0[J + 1, 0, :] + sp_ref[J + 1, 0, :])
    assert d["indirectx"] == ix and d["indirecty"] == iy
    assert ix == STAR["rpstar"] * math.cos(STAR["phi_star"])
    # clearing it gives POT3 alone again
    plan.set_external(None)
    v2, d2 = host_solve(chylib, plan, rho, phi0)
    assert np.array_equal(v2, v) and d2["indirectx"] == 0.0


def test_fp64_chain_matches_oracle(chylib):
    rho, phi0 = density(), phi_start()
    ref, _, _ = oracle_chain(rho, phi0, **STAR)
    plan = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    plan.set_external(**STAR)
    e, _ = host_solve(chylib, plan, rho, phi0)
    assert rel_l2(e, ref) < 1e-12


def test_device_pointers_match_host_pointers(chylib):
    import torch
    rho, phi0 = density(2), phi_start(3)
    plan = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    plan.set_external(**STAR)
    e_host, _ = host_solve(chylib, plan, rho, phi0)
    r = chylib.to_cuda_fortran(rho)
    f = chylib.to_cuda_fortran(phi0)
    plan.solve(r, f)
    torch.cuda.synchronize()
    assert np.array_equal(f.cpu().numpy(), e_host)
    out = chylib.fortran_zeros_cuda((J + 2, K + 2, L))
    plan.star_potential(out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), plan.star_potential())


def test_indirect_shift_per_solve(chylib):
    star = dict(STAR, indirect=True, jmin=2)
    rhos = [density(s) for s in (1, 4, 5)]
    phi0 = phi_start()
    plan = chylib.Plan(chylib.grid(J, K, L), "fp64", 3)
    plain = plan.solve_batch(rhos, [phi0.copy(order="F") for _ in rhos])
    plan.set_external(**star)
    outs, diags = plan.solve_batch(rhos, [phi0.copy(order="F") for _ in rhos], diag=True)
    for rho, v, e, d in zip(rhos, plain, outs, diags):
        ref, sp_ref, (ix, iy) = oracle_chain(rho, phi0, **star)
        check_shift(d, ix, iy, rho, 2, star["mass_star"])
        assert rel_l2(e, ref) < 1e-12
        # STARPHI ~ 1/distance: near the axis a 1e-15 shift of the star moves
        # it by ~1e-13 relative
        assert rel_l2(e - v, sp_ref) < 1e-12
    # STARPHI follows the latest solve
    spn = plan.star_potential()
    assert np.array_equal(outs[-1], plain[-1] + spn)
    refn = oracle_chain(rhos[-1], phi0, **star)[1]
    assert rel_l2(spn, refn) < 1e-12


def test_indirect_jmin_changes_the_moment(chylib):
    rho, phi0 = density(), phi_start()
    plan = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    for jmin in (1, 5, J + 1, J + 2):
        star = dict(STAR, indirect=True, jmin=jmin)
        plan.set_external(**star)
        _, d = host_solve(chylib, plan, rho, phi0)
        _, _, (ix, iy) = oracle_chain(rho, phi0, **star)
        if jmin > J + 1:
            # empty moment: the fixed position over -MASS_STAR, exactly
            assert (d["indirectx"], d["indirecty"]) == (ix, iy)
        else:
            check_shift(d, ix, iy, rho, jmin, star["mass_star"])


def test_solve_multi_applies_each_plans_star(chylib):
    import torch
    rho, phi0 = density(), phi_start()
    a = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    b = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    b.set_external(**STAR)
    r = chylib.to_cuda_fortran(rho)
    fa, fb = chylib.to_cuda_fortran(phi0), chylib.to_cuda_fortran(phi0)
    chylib.solve_multi([a, b], [r, r], [fa, fb])
    torch.cuda.synchronize()
    assert np.array_equal(fb.cpu().numpy(), fa.cpu().numpy() + b.star_potential())


def test_argument_checks(chylib):
    plan = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    with pytest.raises(chylib.ChyError) as e:
        plan.star_potential()
    assert e.value.status == 13   # CHY_ERR_NOT_SETUP: no external potential set
    with pytest.raises(chylib.ChyError):
        plan.set_external(1.0, indirect=True, jmin=0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_binary_companion_is_the_reference_expression(chylib, ora, precision):
    """The BINARY build's companion (pot/ExternalPot.f:57-69, orbit of
    radhydro/ExternalRoutines.f:91-105) with the reference's MASSBIN = 1,
    ABIN = 100: PHI with star and companion equals the oracle's ExternalPot
    (STARPHI, then the companion term, in the reference's order) applied to
    the same solve's PHI without them, bit for bit in every cell, through
    host and device pointers; STARPHI itself is unchanged."""
    import torch
    rho, phi0 = density(3), phi_start(5)
    plan = chylib.Plan(chylib.grid(J, K, L), precision, 1)
    v, _ = host_solve(chylib, plan, rho, phi0)
    plan.set_external(**STAR)
    sp0 = plan.star_potential()
    plan.set_binary(1.0, 100.0)
    e, _ = host_solve(chylib, plan, rho, phi0)
    o = ora.Oracle(J, K, L, nthreads=8)
    o.set_grid(1.0 / J, 0.5 / K)
    o.phi[...] = v
    sp, _ = o.external_pot(**STAR, binary=True, mass_bin=1.0, a_bin=100.0)
    assert np.array_equal(e, np.array(o.phi))
    assert np.array_equal(plan.star_potential(), sp0) and np.array_equal(sp0, sp)
    assert not np.array_equal(e, v + sp)          # the companion term is there
    ed = plan.solve(chylib.to_cuda_fortran(rho), chylib.to_cuda_fortran(phi0))
    torch.cuda.synchronize()
    assert np.array_equal(ed.cpu().numpy(), e)
    plan.set_binary(None)
    f, _ = host_solve(chylib, plan, rho, phi0)
    assert np.array_equal(f, v + sp)
