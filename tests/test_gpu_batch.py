"""Uneven-size batches (the batched workload: densities with JMAX in
{64,128,256}, KMAX in {32,64,128}, LMAX in {64,128,256}, random surface-density
slope and scale height) through chy_solve_multi: every result equals the same
density solved alone, bitwise; the whole batch replays from a captured CUDA
graph with the same results; and the mixed path stays within rel. L2 1e-10 of
the FP64 path."""
import pytest

from chymera_uo_b200 import synth

pytestmark = pytest.mark.gpu

N = 16


def _plans(chy, dens, precision, max_batch):
    cache, out = {}, []
    for _, g in dens:
        key = (g.jmax, g.kmax, g.lmax)
        if key not in cache:
            cache[key] = chy.Plan(chy.grid(*key), precision, max_batch)
        out.append(cache[key])
    return out, cache


def _rel(a, b, J, K):
    import torch
    a, b = a[: J + 1, : K + 1], b[: J + 1, : K + 1]
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def test_uneven_batch_alone_in_the_mix_and_from_a_graph(chylib):
    import torch
    dens = [synth.config_density(4, i) for i in range(N)]
    assert len({(g.jmax, g.kmax, g.lmax) for _, g in dens}) >= 6
    rhos = [chylib.to_cuda_fortran(r) for r, _ in dens]
    plans, cache = _plans(chylib, dens, "mixed", 4)
    mix = chylib.solve_multi(plans, rhos)
    torch.cuda.synchronize()
    for p, r, m in zip(plans, rhos, mix):
        alone = p.solve(r)
        torch.cuda.synchronize()
        assert torch.equal(alone, m)

    outs = [chylib.fortran_zeros_cuda(p.shape) for p in plans]
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        chylib.solve_multi(plans, rhos, outs)
    for _ in range(2):
        for o in outs:
            o.zero_()
        graph.replay()
        torch.cuda.synchronize()
        for o, m in zip(outs, mix):
            assert torch.equal(o, m)

    plans64, _ = _plans(chylib, dens, "fp64", 4)
    ref = chylib.solve_multi(plans64, rhos)
    torch.cuda.synchronize()
    for (rho, g), m, f in zip(dens, mix, ref):
        assert _rel(m, f, g.jmax, g.kmax) <= 1e-10

    # one density of each size class against the oracle
    import numpy as np
    from oracle import oracle as O
    seen = set()
    for (rho, g), m in zip(dens, mix):
        key = (g.jmax, g.kmax, g.lmax)
        if key in seen:
            continue
        seen.add(key)
        oref = np.array(O.Oracle(*key, nthreads=8).solve(rho))
        got = m.cpu().numpy()
        ws = (slice(0, g.jmax + 1), slice(0, g.kmax + 1))
        assert np.linalg.norm((got[ws] - oref[ws]).ravel()) <= 1e-10 * np.linalg.norm(oref[ws].ravel()), key


@pytest.mark.parametrize("precision", ["mixed", "blktri"])
def test_autotuned_schedule_keeps_results_bitwise(chylib, precision):
    """chy_autotune_multi only changes how the work is launched (grids in
    flight, solves per launch sequence, persistent CTAs, the BLKTRI stage
    schedule), never what a solve computes: results after tuning, and from a
    graph captured after it, equal the default schedule's bit for bit."""
    import torch
    dens = [synth.config_density(4, i) for i in range(8)]
    rhos = [chylib.to_cuda_fortran(r) for r, _ in dens]
    plans, cache = _plans(chylib, dens, precision, 4)
    ref = chylib.solve_multi(plans, rhos)
    torch.cuda.synchronize()
    tune = chylib.autotune_multi(plans, rhos, repeats=2)
    assert tune["candidates"] >= 3 and tune["ms"] <= tune["ms_default"]
    assert tune["streams"] in (1, 2, 4, 8) and tune["blk_warps"] in (4, 8, 16)
    assert tune["blk_warps"] * tune["blk_ctas_per_sm"] <= 16 and tune["mode_ctas"] >= 1
    got = chylib.solve_multi(plans, rhos)
    torch.cuda.synchronize()
    for a, b in zip(got, ref):
        assert torch.equal(a, b)
    outs = [chylib.fortran_zeros_cuda(p.shape) for p in plans]
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        chylib.solve_multi(plans, rhos, outs)
    graph.replay()
    torch.cuda.synchronize()
    for a, b in zip(outs, ref):
        assert torch.equal(a, b)
