"""SOURCE's potential, pressure and rotation terms (radhydro/source.f:45-81)
on the GPU through the C ABI (chy_source, and chy_source_binary for a BINARY
build), against the oracle's restatement.

Every cell is computed independently with each operation rounded as the
reference rounds it, so S, T and A must equal the oracle's bit for bit: for
hydro grids equal to and smaller than the potential grid, for JMIN below,
at and above 2, and on the PHI of a real solve with the external potential
added (the reference's order: POT3, ExternalPot, SOURCE).
"""
import numpy as np
import pytest

from chymera_uo_b200 import synth

pytestmark = pytest.mark.gpu

J, K, L = 64, 32, 64


def fields(jh, kh, seed):
    rng = np.random.default_rng(seed)
    f = lambda shape, scale=1.0, off=0.0: np.asfortranarray(off + scale * rng.random(shape))
    hs = (jh + 2, kh + 2, L)
    return dict(omega=f(hs, 2.0, -1.0), p=f(hs, 1e-3), s=f(hs, 1.0, -0.5), t=f(hs, 1.0, -0.5), a=f(hs, 1.0, -0.5))


def run_both(chylib, plan, rho, phi, hyd, delt, jmin, binary=None):
    """chy_source (chy_source_binary with `binary`) on the GPU and the oracle
    on the same arrays; the plan's spacings, R(J) = (J-2) ROF3N and
    RHF(J) = R(J) + ROF3N/2."""
    from oracle import oracle as O
    d = {k: chylib.to_cuda_fortran(v) for k, v in hyd.items()}
    gbin = None if binary is None else dict(binary, u=chylib.to_cuda_fortran(binary["u"]))
    plan.source(chylib.to_cuda_fortran(rho), chylib.to_cuda_fortran(phi), d["omega"], d["p"], d["s"], d["t"],
                d["a"], delt, jmin=jmin, binary=gbin)
    import torch
    torch.cuda.synchronize()
    ref = {k: v.copy(order="F") for k, v in hyd.items()}
    g = plan.grid
    r = np.array([(j - 2) * g.rof3n for j in range(1, J + 3)])
    obin = None if binary is None else dict(binary, rhf=r + g.rof3n / 2.0)
    O.source(r, rho, phi, ref["omega"], ref["p"], ref["s"], ref["t"], ref["a"], delt, g.rof3n, g.zof3n,
             2.0 * 3.1415926535897932 / L, jmin=jmin, binary=obin)
    return {k: d[k].cpu().numpy() for k in ("s", "t", "a")}, ref


@pytest.mark.parametrize("jh,kh", [(J, K), (48, 24), (1, 1)])
@pytest.mark.parametrize("jmin", [1, 2, 5])
@pytest.mark.parametrize("spacing", ["pow2", "general"])
def test_source_bitwise(chylib, jh, kh, jmin, spacing):
    # the default spacings 1/JMAX and 0.5/KMAX are powers of two (the kernel
    # multiplies by their exact reciprocals); 0.3/JMAX and 0.7/KMAX are not
    # (it divides)
    kw = {} if spacing == "pow2" else dict(rof3n=0.3 / J, zof3n=0.7 / K)
    plan = chylib.Plan(chylib.grid(J, K, L, **kw), "fp64", 1)
    rng = np.random.default_rng(11)
    rho = np.asfortranarray(rng.random((J + 2, K + 2, L)))
    phi = np.asfortranarray(-1.0 - rng.random((J + 2, K + 2, L)))
    hyd = fields(jh, kh, 5)
    got, ref = run_both(chylib, plan, rho, phi, hyd, 3.7e-4, jmin)
    for k in ("s", "t", "a"):
        assert np.array_equal(got[k], ref[k]), k
    if jh >= 2:
        # cells outside the loops keep their values
        assert np.array_equal(got["t"][:, 0, :], hyd["t"][:, 0, :])
        assert np.array_equal(got["a"][:, kh + 1, :], hyd["a"][:, kh + 1, :])


@pytest.mark.parametrize("jh,kh", [(J, K), (48, 24)])
@pytest.mark.parametrize("jmin", [1, 2, 5])
def test_source_binary_bitwise(chylib, jh, kh, jmin):
    """The BINARY build's terms (radhydro/source.f:61-62, 76-77) with
    getBinaryPosition's OMEGABIN: S and A bitwise the oracle's, T as in a
    BINARY = 0 build, and S, A differing from the BINARY = 0 results."""
    plan = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    rng = np.random.default_rng(13)
    rho = np.asfortranarray(rng.random((J + 2, K + 2, L)))
    phi = np.asfortranarray(-1.0 - rng.random((J + 2, K + 2, L)))
    hyd = fields(jh, kh, 7)
    u = np.asfortranarray(rng.random(hyd["omega"].shape) - 0.5)
    # a close companion, so that its terms are visible in S and A
    binary = dict(u=u, mass_star=1.0, mass_bin=0.5, a_bin=1.5)
    got, ref = run_both(chylib, plan, rho, phi, hyd, 3.7e-4, jmin, binary=binary)
    for k in ("s", "t", "a"):
        assert np.array_equal(got[k], ref[k]), k
    plain, _ = run_both(chylib, plan, rho, phi, hyd, 3.7e-4, jmin)
    assert np.array_equal(got["t"], plain["t"])
    for k in ("s", "a"):
        assert not np.array_equal(got[k], plain[k]), k


def test_source_after_solve_and_external_potential(chylib):
    import torch
    rho = synth.disk_density(J, K, L, 1, spiral=True, spectrum=True)
    plan = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    plan.set_external(1.0, 0.0125, 0.0031, 0.7)
    r = chylib.to_cuda_fortran(rho)
    f = chylib.fortran_zeros_cuda((J + 2, K + 2, L))
    plan.solve(r, f)
    torch.cuda.synchronize()
    phi = f.cpu().numpy()
    hyd = fields(J, K, 9)
    got, ref = run_both(chylib, plan, rho, phi, hyd, 1e-3, 2)
    for k in ("s", "t", "a"):
        assert np.array_equal(got[k], ref[k]), k
    # the gravity term dominates T near the midplane: sign check on a physical field
    assert np.isfinite(got["t"]).all()


def test_source_argument_checks(chylib):
    import torch
    plan = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    big = chylib.fortran_zeros_cuda((J + 4, K + 2, L))
    x = chylib.fortran_zeros_cuda((J + 2, K + 2, L))
    with pytest.raises(chylib.ChyError) as e:
        plan.source(x, x, big, big, big, big, big, 1e-3)
    assert e.value.status == 11   # CHY_ERR_DIMS: hydro grid larger than the plan's
    with pytest.raises(chylib.ChyError):
        plan.source(x, x, x, x, x, x, x, 1e-3, jmin=0)
    with pytest.raises(chylib.ChyError) as e:
        plan.source(x, x, x, x, x, x, x, 1e-3, binary=dict(u=x, mass_star=1.0, a_bin=0.0))
    assert e.value.status == 10   # CHY_ERR_ARG: the separation must be positive
    torch.cuda.synchronize()
