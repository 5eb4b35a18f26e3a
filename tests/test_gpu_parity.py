"""libchy_pot3 on the GPU against the CPU oracle, through the C ABI.

Tolerances (relative L2 over every cell of the write set):
  * plain FP64 path: 1e-12 at 64x32x64.  At 256x128x256 the oracle's own
    BLKTRI solve of the m = 0 mode is only accurate to ~2.4e-12 (measured
    against a long-double-refined solution in tests/test_oracle.py), so the
    bar there is 5e-12; the FP64 path itself is ~10x closer to the exact
    solution than the oracle.
  * mixed path (FP16 hi/lo tensor-core transforms, FP32 sweeps, FP64
    refinement): 1e-10.
"""
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
def oracle_result(cfg, literal="gcc", isym=2, maxtrm=10, redge=0.0, npoint=8, seed_override=None):
    from oracle import oracle as O
    if seed_override is None:
        rho, g = synth.config_density(cfg)
    else:
        J, K, L = cfg
        rho, g = synth.disk_density(J, K, L, seed_override, spiral=True, spectrum=True), synth.default_grid(J, K, L)
    o = O.Oracle(g.jmax, g.kmax, g.lmax, literal_r8=(literal == "r8"), nthreads=8, want_coef=True)
    phi = o.solve(rho, isym=isym, maxtrm=maxtrm, redge=redge, npoint=npoint)
    coef = np.array(o.coef)
    return rho, phi, o.inside(), coef


def gpu_solve(chy, rho, J, K, L, precision="fp64", phi0=None, **gkw):
    plan = chy.Plan(chy.grid(J, K, L, **gkw), precision, 1)
    phi = phi0.copy(order="F") if phi0 is not None else np.zeros_like(rho, order="F")
    (out,), (d,) = plan.solve_batch([rho], [phi], diag=True)
    return out, d, plan


@pytest.mark.parametrize("literal", ["gcc", "r8"])
def test_fp64_small_grid(chylib, literal):
    rho, ref, dref, _ = oracle_result(1, literal)
    phi, d, _ = gpu_solve(chylib, rho, 64, 32, 64, "fp64", literal=literal)
    ws = write_set(64, 32)
    assert rel_l2(phi[ws], ref[ws]) < 1e-12
    assert abs(d["tmass"] - dref["tmass"]) <= 1e-13 * dref["tmass"]
    assert d["klocat"] == dref["klocat"]
    assert abs(d["phichk"] - dref["phichk"]) <= 1e-4 * abs(dref["phichk"])


def test_fp64_large_grid(chylib):
    rho, ref, dref, _ = oracle_result(2)
    phi, d, _ = gpu_solve(chylib, rho, 256, 128, 256, "fp64")
    ws = write_set(256, 128)
    assert rel_l2(phi[ws], ref[ws]) < 5e-12
    assert abs(d["tmass"] - dref["tmass"]) <= 1e-13 * dref["tmass"]


@pytest.mark.parametrize("cfg", [1, 2, 3])
def test_mixed_meets_1e10(chylib, cfg):
    rho, ref, dref, _ = oracle_result(cfg)
    g = synth.config_density(cfg)[1]
    phi, d, _ = gpu_solve(chylib, rho, g.jmax, g.kmax, g.lmax, "mixed")
    ws = write_set(g.jmax, g.kmax)
    assert rel_l2(phi[ws], ref[ws]) < 1e-10
    assert d["iterations"] >= 1 and d["corr_rel"][0] == pytest.approx(1.0)


@pytest.mark.parametrize("J,K,L", [(256, 128, 64), (64, 32, 64), (80, 32, 64), (192, 64, 32)])
def test_mixed_mode_kernels(chylib, J, K, L):
    """The two fused mode-solve kernels -- k_mode_pair (a CTA pair per mode,
    two modes per SM, the sweeps' meeting rows and the iterate's edge column
    exchanged through distributed shared memory) and k_mode_mixed (one CTA
    per mode) -- take every power-of-two scale per radial half and give the
    same bits; both meet 1e-10 against the oracle.  A mode's result does not
    depend on the batch around it or on which CTAs solved it."""
    rho, ref, _, _ = oracle_result((J, K, L), seed_override=17)
    rho2 = synth.disk_density(J, K, L, 18, spiral=True, spectrum=True)
    ws = write_set(J, K)
    outs = {}
    for mk, kernel in ((2, 2), (1, 1), (0, 1)):
        plan = chylib.Plan(chylib.grid(J, K, L), "mixed", 3)
        plan.set_schedule(mode_kernel=mk)
        (single,), (d,) = plan.solve_batch([rho], diag=True)
        # mode_kernel 0 (automatic) keeps one CTA per mode for so few modes
        assert chylib.lib().chy_dbg_mixed_kernel(plan._p) == kernel
        assert rel_l2(single[ws], ref[ws]) < 1e-10
        assert d["iterations"] == 2 and d["corr_rel"][0] == pytest.approx(1.0) and d["corr_rel"][1] < 1e-5
        batch = plan.solve_batch([rho, rho2, rho])
        assert np.array_equal(batch[0], single) and np.array_equal(batch[2], single)
        outs[mk] = single
    assert np.array_equal(outs[2], outs[1]) and np.array_equal(outs[0], outs[1])


def test_mixed_automatic_kernel_choice(chylib):
    """mode_kernel 0 runs k_mode_pair once the launch holds at least 16 modes
    per group of warps (32 per CTA pair) and one CTA per mode below that;
    the results are the same bits either way."""
    import torch
    J, K, L = 64, 32, 256
    g = chylib.grid(J, K, L)
    rhos = [chylib.to_cuda_fortran(synth.disk_density(J, K, L, 40 + i, spiral=True, spectrum=True)) for i in range(20)]
    plan = chylib.Plan(g, "mixed", 20)
    small = plan.solve_batch(rhos[:1])
    torch.cuda.synchronize()
    assert chylib.lib().chy_dbg_mixed_kernel(plan._p) == 1
    big = plan.solve_batch(rhos)              # 20 x 256 modes >= 32 x 74 pairs
    torch.cuda.synchronize()
    assert chylib.lib().chy_dbg_mixed_kernel(plan._p) == 2
    assert torch.equal(small[0], big[0])


def test_mixed_refinement_converges_geometrically(chylib):
    rho, ref, _, _ = oracle_result(3)
    ws = write_set(256, 128)
    errs = []
    for corrections in (0, 1, 2):
        plan = chylib.Plan(chylib.grid(256, 128, 256), "mixed", 1)
        plan.set_refine(corrections)
        (phi,), (d,) = plan.solve_batch([rho], diag=True)
        errs.append(rel_l2(phi[ws], ref[ws]))
        assert len(d["corr_rel"]) == corrections + 1 or corrections == 0
    assert errs[0] < 1e-4 and errs[1] < errs[0] * 1e-3 and errs[2] < 1e-11


def test_write_set_and_untouched_cells(chylib):
    """Only the reference's write set changes: PHI(:,KMAX+2,:) and
    PHI(JMAX+2,1,:) keep the caller's values (radhydro/3dhyd-main.f:457-465
    zeroes them; POT3/BDYGEN never write them)."""
    rho, ref, _, _ = oracle_result(1)
    J, K = 64, 32
    phi0 = np.full_like(rho, 7.0, order="F")
    for prec in ("fp64", "mixed"):
        phi, _, plan = gpu_solve(chylib, rho, J, K, 64, prec, phi0=phi0)
        assert np.all(phi[:, K + 1, :] == 7.0)
        assert np.all(phi[J + 1, 0, :] == 7.0)
        assert np.all(np.isfinite(phi))
        # the device-pointer path writes the same cells with the same values
        import torch
        rd = chylib.to_cuda_fortran(rho)
        pd = chylib.to_cuda_fortran(phi0)
        plan.solve(rd, pd)
        torch.cuda.synchronize()
        assert np.array_equal(pd.cpu().numpy(), phi)


def test_boundary_modes_match_oracle_bdygen(chylib):
    """X at the boundary = POT3's transform of BDYGEN's boundary values."""
    from oracle import oracle as O
    rho, g = synth.config_density(1)
    J, K, L = 64, 32, 64
    o = O.Oracle(J, K, L)
    o.set_grid(1.0 / J, 0.5 / K); o.rho[...] = rho; o.phi[...] = 0.0
    o.setbdy(0, 2); o.bdygen(10, 2, 0.0)
    pb = np.array(o.phi)
    plan = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    plan.solve_batch([rho])
    X = plan.debug_work("X", L * K * J).reshape(L, K, J)
    for (j, k) in [(0, K - 1), (J // 2, K - 1), (J - 1, K - 1), (J - 1, 0), (J - 1, K // 2)]:
        ref = O.forward_real(pb[j + 1, k + 1, :].copy(), False)
        assert np.abs(X[:, k, j] - ref).max() <= 1e-14 * np.abs(ref).max()


@pytest.mark.parametrize("isym,maxtrm,npoint,redge", [(1, 10, 8, 0.0), (3, 8, 8, 0.0), (2, 4, 7, 0.0),
                                                      (-2, 10, 8, 0.0), (2, 10, 8, 0.6)])
def test_call_parameter_variants(chylib, isym, maxtrm, npoint, redge):
    """ISYM, MAXTRM, NPOINT and REDGE as BDYGEN/ZAXPHI accept them
    (pot/boundary.f:97-105, pot/pot3.f:328-348)."""
    rho, ref, dref, _ = oracle_result(1, "gcc", isym, maxtrm, redge, npoint)
    phi, d, _ = gpu_solve(chylib, rho, 64, 32, 64, "fp64", isym=isym, maxtrm=maxtrm, npoint=npoint, redge=redge)
    ws = write_set(64, 32)
    assert rel_l2(phi[ws], ref[ws]) < 1e-12
    assert abs(d["tmass"] - dref["tmass"]) <= 1e-12 * abs(dref["tmass"])


# JMAX = 80 and 208 are multiples of 16 but not of 64: the mixed path's tiles
# then run past JMAX (half tiles zero-filled, whole chunks empty)
@pytest.mark.parametrize("J,K,L", [(128, 64, 128), (64, 32, 256), (256, 64, 64), (80, 32, 64), (208, 64, 128)])
def test_other_grid_sizes(chylib, J, K, L):
    rho, ref, _, _ = oracle_result((J, K, L), seed_override=21)
    for prec, tol in (("fp64", 2e-12), ("mixed", 1e-10)):
        phi, _, _ = gpu_solve(chylib, rho, J, K, L, prec)
        ws = write_set(J, K)
        assert rel_l2(phi[ws], ref[ws]) < tol, prec


def test_copy_paths_match_tensor_map_paths(chylib):
    """The transforms read RHO and X through tensor-map tiles when rows are
    16-byte aligned and JMAX is even, else through 8-byte copies:
      * JMAX = 65 runs the copy paths of both transforms, held to the oracle
        like the other grid sizes;
      * an RHO array 8 bytes past a 16-byte boundary runs the forward
        transform's copy path, and PHI equals the aligned array's bit for bit."""
    import torch
    J, K, L = 65, 32, 64
    rho, ref, _, _ = oracle_result((J, K, L), seed_override=23)
    phi, _, _ = gpu_solve(chylib, rho, J, K, L, "fp64")
    ws = write_set(J, K)
    assert rel_l2(phi[ws], ref[ws]) < 2e-12
    J, K, L = 64, 32, 64
    rho = synth.disk_density(J, K, L, 3, spiral=True, spectrum=True)
    for prec in ("fp64", "mixed"):
        plan = chylib.Plan(chylib.grid(J, K, L), prec, 1)
        a = chylib.to_cuda_fortran(rho)
        flat = torch.zeros(rho.size + 1, dtype=torch.float64, device="cuda")
        u = flat[1:].view(L, K + 2, J + 2).permute(2, 1, 0)
        u.copy_(a)
        assert u.data_ptr() % 16 == 8
        pa, pu = plan.solve(a), plan.solve(u)
        torch.cuda.synchronize()
        assert torch.equal(pa, pu), prec


def test_batch_results_equal_single_solves_bitwise(chylib):
    """Each result is the same alone and in a batch: every reduction has a
    fixed order, nothing depends on scheduling."""
    import torch
    J, K, L = 64, 32, 64
    rhos = [synth.disk_density(J, K, L, s, spiral=True, spectrum=True) for s in range(5)]
    for prec in ("fp64", "mixed"):
        plan = chylib.Plan(chylib.grid(J, K, L), prec, 8)
        rd = [chylib.to_cuda_fortran(r) for r in rhos]
        batch = plan.solve_batch(rd)
        torch.cuda.synchronize()
        for r, b in zip(rd, batch):
            single = plan.solve(r)
            torch.cuda.synchronize()
            assert torch.equal(single, b)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_host_pipeline_equals_device_path(chylib, prec):
    """Host-pointer batches run through the staged copy-in / solve / copy-out
    pipeline; with more chunks than staging slots every slot is reused, and
    every result still equals the device-pointer solve bit for bit, with the
    caller's untouched cells kept per solve."""
    import torch
    J, K, L = 64, 32, 64
    n = 11
    rhos = [synth.disk_density(J, K, L, 40 + s, spiral=True, spectrum=True) for s in range(n)]
    phis = [np.full_like(r, float(i + 1), order="F") for i, r in enumerate(rhos)]
    plan = chylib.Plan(chylib.grid(J, K, L), prec, 2)      # chunks of 2 solves, 3 slots
    out = plan.solve_batch(rhos, phis)
    dev = plan.solve_batch([chylib.to_cuda_fortran(r) for r in rhos],
                           [chylib.to_cuda_fortran(f) for f in [np.full_like(r, float(i + 1), order="F")
                                                                for i, r in enumerate(rhos)]])
    torch.cuda.synchronize()
    for i, (h, d) in enumerate(zip(out, dev)):
        assert np.array_equal(h, d.cpu().numpy()), i
        assert np.all(h[:, K + 1, :] == i + 1) and np.all(h[J + 1, 0, :] == i + 1)
    _, diags = plan.solve_batch(rhos[:5], [np.zeros_like(r, order="F") for r in rhos[:5]], diag=True)
    assert all(d["tmass"] > 0 for d in diags)


def test_coef_diagnostics(chylib):
    """/COEFS/ amplitude and phase (pot/pot3.f:105-132)."""
    import torch
    rho, _, _, coef_ref = oracle_result(1)
    J, K, L = 64, 32, 64
    plan = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
    coef = torch.zeros((2, L // 2, K + 2, J + 2), dtype=torch.float64, device="cuda").permute(3, 2, 1, 0)
    plan.set_coef(coef)
    plan.solve(chylib.to_cuda_fortran(rho))
    torch.cuda.synchronize()
    got = coef.cpu().numpy()
    sel = (slice(1, J + 1), slice(1, K + 1))
    amp, ph = got[sel + (slice(None), 0)], got[sel + (slice(None), 1)]
    amp_r, ph_r = coef_ref[sel + (slice(None), 0)], coef_ref[sel + (slice(None), 1)]
    assert np.abs(amp - amp_r).max() <= 1e-9 * np.abs(amp_r).max()
    # COEF(J,K,N,2) holds A1(1), the raw m = 0 coefficient
    assert np.abs(ph[..., -1] - ph_r[..., -1]).max() <= 1e-12 * np.abs(ph_r[..., -1]).max()
    # a phase is only as well defined as its amplitude: an error e in the
    # transform moves it by ~e/amplitude radians, so compare where the
    # amplitude (relative to m = 0) is above 1e-6, modulo 360 degrees
    mask = amp_r[..., :-1] > 1e-6
    d = np.abs(ph[..., :-1] - ph_r[..., :-1])[mask]
    d = np.minimum(d, np.abs(d - 360.0))
    assert mask.sum() > 1000 and d.max() <= 1e-4


def test_tensor_core_tile_product(chylib):
    """One tcgen05 tile product (FP16 hi/lo, three passes) against FP64, with
    the plan's resident eigenbasis tile read as Q^T (K-major descriptor) and
    as Q (the transposed, MN-major descriptor)."""
    import ctypes as C
    import torch
    J, K, L = 256, 128, 256
    g = chylib.grid(J, K, L)
    plan = chylib.Plan(g, "mixed", 1)
    NZ = K - 1
    out = np.zeros(NZ * NZ)
    chylib.lib().chy_dbg_table(C.byref(g), b"Qt", out.ctypes.data_as(C.POINTER(C.c_double)), NZ * NZ)
    Qt = out.reshape(NZ, NZ)
    for which, A in ((0, Qt), (1, Qt.T)):
        for NT in (64, 256):
            Bm = np.zeros((NT, 128), np.float32)
            Bm[:, :NZ] = np.random.default_rng(NT).uniform(-2000, 2000, (NT, NZ))
            Bd = torch.from_numpy(Bm).cuda()
            Dd = torch.zeros((128, NT), dtype=torch.float32, device="cuda")
            assert chylib.lib().chy_dbg_umma(plan._p, which, Bd.data_ptr(), Dd.data_ptr(), NT) == 0
            ref = np.zeros((128, 128)); ref[:NZ, :NZ] = A
            ref = 4096.0 * ref @ Bm.astype(np.float64).T
            assert np.abs(Dd.cpu().numpy() - ref).max() <= 5e-6 * np.abs(ref).max(), (which, NT)


def test_status_codes_on_device(chylib):
    import ctypes as C
    L = chylib.lib()
    p = C.c_void_p()
    g = chylib.grid(64, 48, 64)     # KMAX not a power of two
    assert L.chy_plan_create(C.byref(g), 0, 1, C.byref(p)) == 2
    g = chylib.grid(64, 32, 64)
    assert L.chy_plan_create(C.byref(g), 0, 1, C.byref(p)) == 0
    assert L.chy_solve(p, None, None, None, 0, None) == 10
    L.chy_plan_destroy(p)


@pytest.mark.parametrize("prec", ["blktri", "fp64"])
def test_iprint_report_text(chylib, prec):
    """chy_plan_report: the IPRINT = 1 unit-3 text (pot/pot3.f:402-418) of the
    latest solve equals the reference's edit descriptors applied to the
    oracle's PHAC and COEF: character for character except PHAC's values,
    which are compared within their printed precision (tests/unit3.py)."""
    import sys, os
    import torch
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from unit3 import check, report
    from oracle import oracle as O
    rho, g = synth.config_density(1)
    J, K, L = 64, 32, 64
    o = O.Oracle(J, K, L, nthreads=8, want_coef=True)
    o.solve(rho)
    plan = chylib.Plan(chylib.grid(J, K, L), prec, 1)
    with pytest.raises(chylib.ChyError):
        plan.report()                      # no COEF output set
    coef = torch.zeros((2, L // 2, K + 2, J + 2), dtype=torch.float64, device="cuda").permute(3, 2, 1, 0)
    plan.set_coef(coef)
    plan.solve(chylib.to_cuda_fortran(rho))
    check(plan.report(), report(lambda k: o.phac[k - 1], o.coef, J, K, L))


def test_fp64_paths_against_a_long_double_mode_solution(chylib, ora):
    """At 256x128x256 the m = 0 mode system, with the device's right-hand side
    (the oracle's forward transform, bitwise the device's, and the device's
    boundary rows, folded in POT3's order), solved by sparse LU and refined
    with long-double residuals: the FP64 eigenbasis path's mode is within
    1e-12 of it (it is ~10x closer than BLKTRI's own rounding), and the
    BLKTRI-order path's mode is within BLKTRI's 5e-12 floor."""
    import ctypes as C
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    J, K, L = 256, 128, 256
    M, NZ = J - 1, K - 1
    rho, _ = synth.config_density(2)
    g = chylib.grid(J, K, L)

    def table(name, n):
        out = np.zeros(n)
        assert chylib.lib().chy_dbg_table(C.byref(g), name.encode(), out.ctypes.data_as(C.POINTER(C.c_double)), n) >= 0
        return out

    an, bn, cn = table("an", NZ), table("bn", NZ), table("cn", NZ)
    am, cm = table("am", M), table("cm", M)
    bm = table("blk_bm", L * M)[:M]                       # mode l = 0
    sc = table("scalars", 8)
    pig4, cmmax, cnmax = sc[1], sc[2], sc[4]
    modes = {}
    for prec in ("fp64", "blktri"):
        plan = chylib.Plan(g, prec, 1)
        plan.solve_batch([rho])
        modes[prec] = plan.debug_work("X", L * K * J).reshape(L, K, J)[0]
    X0 = modes["fp64"]
    F0 = np.array([[ora.forward_real(rho[j + 1, k + 1, :].copy(), False)[0] for j in range(M)] for k in range(NZ)])
    y = np.asfortranarray((pig4 * F0).T)
    y[:, NZ - 1] = y[:, NZ - 1] - cnmax * X0[NZ, :M]
    y[M - 1, :] = y[M - 1, :] - cmmax * X0[:NZ, M]
    Tm = sp.diags([am[1:], bm, cm[:-1]], [-1, 0, 1])
    Tn = sp.diags([an[1:], bn, cn[:-1]], [-1, 0, 1])
    A = (sp.kron(Tn, sp.eye(M)) + sp.kron(sp.eye(NZ), Tm)).tocsc()
    lu = spl.splu(A)
    b = y.flatten(order="F")
    x = lu.solve(b)
    Al = A.astype(np.longdouble)
    for _ in range(3):
        r = b.astype(np.longdouble) - Al @ x.astype(np.longdouble)
        x = x + lu.solve(r.astype(np.float64))
    xt = x.reshape((M, NZ), order="F")
    err = {p: float(np.linalg.norm(modes[p][:NZ, :M].T - xt) / np.linalg.norm(xt)) for p in modes}
    assert err["fp64"] < 1e-12, err
    assert err["blktri"] < 5e-12, err
    assert err["fp64"] < err["blktri"], err


@pytest.mark.parametrize("prec", ["mixed", "blktri"])
def test_host_copies_read_and_write_only_their_cells(chylib, prec):
    """Host-pointer solves copy RHO in and PHI out as single linear spans.
    RHO cells outside the read set RHO(2:JMAX, 2:KMAX, :) -- here NaN -- do
    not reach the result, and PHI cells outside the write set (PHI(:, KMAX+2, :)
    and PHI(JMAX+2, 1, :), here random) come back unchanged; the result equals
    the device-pointer solve of a clean RHO, bit for bit, through a plan and
    through the server."""
    import torch
    J, K, L = 64, 32, 64
    clean = synth.disk_density(J, K, L, 23, spiral=True, spectrum=True)
    dirty = clean.copy(order="F")
    dirty[0, :, :] = np.nan          # RHO(1, :, :)
    dirty[J:, :, :] = np.nan         # RHO(JMAX+1:JMAX+2, :, :)
    dirty[:, 0, :] = np.nan          # RHO(:, 1, :)
    dirty[:, K:, :] = np.nan         # RHO(:, KMAX+1:KMAX+2, :)
    rng = np.random.default_rng(4)
    phi0 = np.zeros_like(clean, order="F")
    phi0[:, K + 1, :] = rng.random((J + 2, L))
    phi0[J + 1, 0, :] = rng.random(L)
    plan = chylib.Plan(chylib.grid(J, K, L), prec, 1)
    ref = plan.solve(chylib.to_cuda_fortran(clean), chylib.to_cuda_fortran(phi0))
    torch.cuda.synchronize()
    ref = ref.cpu().numpy()
    host = plan.solve(dirty, phi0.copy(order="F"))
    assert np.array_equal(host, ref)
    assert np.array_equal(host[:, K + 1, :], phi0[:, K + 1, :]) and np.array_equal(host[J + 1, 0, :], phi0[J + 1, 0, :])
    # pinned host arrays: the untouched cells are read through the array's
    # device mapping by a kernel instead of being copied
    pr = chylib.pinned_fortran(dirty.shape)
    pr[...] = dirty
    pp = chylib.pinned_fortran(dirty.shape)
    pp[...] = phi0
    plan.solve(pr, pp)
    assert np.array_equal(np.asarray(pp), ref)
    srv = chylib.Server(prec, hbm_budget=4 << 30, max_batch=2)
    try:
        a = chylib.pinned_fortran(dirty.shape)
        a[...] = dirty
        f = chylib.pinned_fortran(dirty.shape)
        f[...] = phi0
        t = srv.submit(chylib.grid(J, K, L), a, f)
        srv.wait(t)
        assert np.array_equal(np.asarray(f), ref)
    finally:
        srv.close()
