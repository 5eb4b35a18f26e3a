"""The serving loop (chy_server_*): requests of mixed grid sizes arrive on a
Poisson clock while earlier ones are on the GPU; each result must equal the
same density solved alone through a plain plan (bitwise: the kernels reduce in
a fixed order per solve), mixed-precision results stay within rel. L2 1e-10
of the FP64 path and, for one request of each size class, of the oracle, and
requests of one grid share batches.  The mix includes a 512 x 128 x 512
request, which the mixed server solves on its wide pipeline."""
import threading

import numpy as np
import pytest

from chymera_uo_b200 import synth

pytestmark = pytest.mark.gpu

SIZES = [(64, 32, 64), (128, 64, 128), (64, 32, 128), (256, 128, 256), (128, 32, 64), (512, 128, 512)]


def _requests(n, seed=7):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        J, K, L = SIZES[int(rng.integers(len(SIZES)))] if i >= 8 else SIZES[0]
        if i == n - 1:
            J, K, L = SIZES[-1]   # one request of the largest class, at the end of the stream
        rho = synth.disk_density(J, K, L, 10**6 + i, slope=float(rng.uniform(-2, -1)),
                                 h=float(rng.uniform(0.03, 0.1)), spiral=True, spectrum=True)
        out.append(((J, K, L), rho))
    return out


def test_served_results_equal_solves_alone(chylib):
    reqs = _requests(24)
    srv = chylib.Server("mixed", hbm_budget=24 << 30, max_batch=4)
    phis = []
    for (J, K, L), rho in reqs:
        a = chylib.pinned_fortran(rho.shape)
        a[...] = rho
        f = chylib.pinned_fortran(rho.shape)
        f[...] = 3.0
        phis.append((a, f))
    tickets = [None] * len(reqs)
    rng = np.random.default_rng(1)

    def producer():
        import time
        for i, ((J, K, L), _) in enumerate(reqs):
            if i >= 8:    # the first eight arrive at once (one grid), the rest on a Poisson clock
                time.sleep(float(rng.exponential(0.002)))
            tickets[i] = srv.submit(chylib.grid(J, K, L), *phis[i])

    th = threading.Thread(target=producer)
    th.start()
    th.join()
    lat = [srv.wait(t) for t in tickets]
    stats = srv.stats()
    srv.close()
    assert stats["completed"] == len(reqs) and stats["batches"] < len(reqs)
    assert all(x > 0 for x in lat)

    from oracle import oracle as O
    plans, plans64, checked = {}, {}, set()
    for ((J, K, L), rho), (_, f) in zip(reqs, phis):
        key = (J, K, L)
        if key not in plans:
            plans[key] = chylib.Plan(chylib.grid(J, K, L), "mixed", 1)
            plans64[key] = chylib.Plan(chylib.grid(J, K, L), "fp64", 1)
        alone = plans[key].solve(rho, np.full_like(rho, 3.0, order="F"))
        assert np.array_equal(alone, f), key
        ref = plans64[key].solve(rho)
        ws = (slice(0, J + 1), slice(0, K + 1))
        assert np.linalg.norm((f[ws] - ref[ws]).ravel()) <= 1e-10 * np.linalg.norm(ref[ws].ravel())
        assert np.all(f[:, K + 1, :] == 3.0)
        if key not in checked:   # one request per size class against the oracle
            checked.add(key)
            o = O.Oracle(J, K, L, nthreads=8)
            oref = np.array(o.solve(rho))
            assert np.linalg.norm((f[ws] - oref[ws]).ravel()) <= 1e-10 * np.linalg.norm(oref[ws].ravel()), key
    assert (512, 128, 512) in checked


def test_blktri_server_equals_plain_plan(chylib):
    """A server of the BLKTRI-order path returns each request bitwise as a
    plain plan of that path solves it."""
    reqs = _requests(6, seed=3)
    srv = chylib.Server("blktri", hbm_budget=16 << 30, max_batch=2)
    bufs = []
    for (J, K, L), rho in reqs[:5]:
        a = chylib.pinned_fortran(rho.shape)
        a[...] = rho
        f = chylib.pinned_fortran(rho.shape)
        f[...] = 0.0
        bufs.append((a, f))
    tickets = [srv.submit(chylib.grid(J, K, L), a, f) for ((J, K, L), _), (a, f) in zip(reqs[:5], bufs)]
    for t in tickets:
        srv.wait(t)
    srv.close()
    for ((J, K, L), rho), (_, f) in zip(reqs[:5], bufs):
        alone = chylib.Plan(chylib.grid(J, K, L), "blktri", 1).solve(rho)
        assert np.array_equal(alone, f), (J, K, L)
