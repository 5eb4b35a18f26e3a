"""pot3 throughput bench: solves/s of the mixed-precision B200 pot3 at
JMAX x KMAX x LMAX = 256 x 128 x 256 (SETBDY + BDYGEN + POT3 of the
reference, pot/boundary.f and pot/pot3.f), with p50/p99 single-solve latency,
the plain FP64 GPU path on the same inputs, and accuracy against both.

One step = one batched launch sequence over --batch independent seeded disk
densities (m=2 spiral + m<=32 spectrum), inputs and outputs resident in HBM
(B x 137 MB, far larger than the 126 MB L2, so nothing is re-read from L2
across steps).  `e2e` is the same metric through the public API with pinned
host buffers, host<->device copies inside the timed region.

    python bench.py [--gpus N --steps K --warmup W --batch B]
    python bench.py --impl reference      # the CPU restatement on host cores

Multi-GPU (torchrun): every rank solves its own densities; there is no
exchange step in a pot3 solve, so ranks are replicas (weak scaling), timed
between barriers with the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

J, K, L = 256, 128, 256
METRIC = "pot3 solves/s @256x128x256 mixed vs FP64 (rel L2≤1e-10); p50/p99 latency"
UNIT = "solves/s"
WORKLOAD = "pot3 256x128x256 mixed precision, seeded disks: m=2 spiral + m<=32 spectrum"
SEED0 = 3
SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")


def densities(n, first):
    from chymera_uo_b200 import synth
    return [synth.disk_density(J, K, L, SEED0 + 7919 * (first + i), spiral=True, spectrum=True)
            for i in range(n)]


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- helpers
# Replicas: every rank solves its own densities; the only collectives are the
# barriers around the timed region and the max of the ranks' times.
def init_replicas(ws, local, backend="nccl", timeout_s=120):
    """The process group for ws > 1 ranks (None for one rank)."""
    if ws <= 1:
        return None
    import datetime
    import torch
    import torch.distributed as dist
    kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return dist


def replica_barrier(dist, device):
    import torch
    if dist is not None:
        dist.barrier()
    if device == "cuda":
        torch.cuda.synchronize()


def replica_max(dist, x, device):
    """Max of x over the ranks (the slowest rank's time)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(ws, solves_per_rank_step, steps, ms_max):
    """Whole-job solves/s: all ranks' solves over the slowest rank's time."""
    return ws * solves_per_rank_step * steps / (ms_max * 1e-3)


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), ws


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={SMI_FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.index)], stdout=self.out, stderr=subprocess.DEVNULL)
            t0 = time.time()
            while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.05)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.out.close()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), float(f[3]), f[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        busy = [r for r in rows if r[2] > 200.0] or rows
        reasons = sorted({REASONS[i] for r in busy for i, v in enumerate(r[3]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median([r[0] for r in busy])), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(busy),
                "power_w_median": float(np.median([r[2] for r in busy]))}


def peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic_per_solve():
    """DRAM bytes (read + write) per solve of the mode-solve kernel from the
    committed ncu summary of that kernel, or None."""
    path = os.path.join(HERE, "profiles", "k_mode_mixed_256x128x256.md")
    try:
        m = re.search(r"dram_bytes_per_solve:\s*([0-9]+)", open(path).read())
    except OSError:
        return None
    return int(m.group(1)) if m else None


def mode_solve_bytes_per_solve():
    """Algorithmic HBM bytes of the mode-solve kernel per solve: it reads the
    transformed right-hand side X (LMAX x KMAX x JMAX doubles, the boundary
    row and column included) once and writes the interior modes
    (LMAX x (KMAX-1) x (JMAX-1) doubles) once."""
    return 8 * L * K * J + 8 * L * (K - 1) * (J - 1)


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    rank, _, ws = dist_info()
    if rank != 0:
        return 0
    from oracle import oracle as O
    cores = host_threads()
    rho = densities(1, 0)[0]
    o = O.Oracle(J, K, L, literal_r8=False, nthreads=cores)
    for _ in range(args.warmup):
        o.solve(rho)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.solve(rho)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = args.steps / total
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOAD.replace("mixed precision", "FP64 CPU restatement"),
                       "jmax": J, "kmax": K, "lmax": L, "solves_per_step": 1, "parallelism": "openmp"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{args.steps} timed solves (1 per step) of one 256x128x256 disk, "
                                       f"SETBDY+BDYGEN+POT3, {cores} OpenMP threads, gcc -O2 "
                                       "-ffp-contract=off"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "latency_ms": {"p50": 1e3 * float(np.median(times)),
                           "p99": 1e3 * float(np.percentile(times, 99)), "samples": len(times)}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- CPU baseline (rank 0, N=1)
def cpu_baseline(rhos, budget_s, max_solves):
    """Times the oracle port on host cores over a bounded sample; returns the
    record and its outputs (used to check the GPU results)."""
    from oracle import oracle as O
    cores = host_threads()
    o = O.Oracle(J, K, L, literal_r8=False, nthreads=cores)
    outs, t = [], 0.0
    for rho in rhos[:max_solves]:
        t0 = time.perf_counter()
        phi = o.solve(rho)
        t += time.perf_counter() - t0
        outs.append(np.array(phi))
        if t >= budget_s and len(outs) >= 2:
            break
    rec = {"value": len(outs) / t, "unit": UNIT, "cores": cores, "kind": "port",
           "sample": f"{len(outs)} solves of the bench's first densities (256x128x256, SETBDY+BDYGEN+POT3), "
                     f"{t:.1f} s, {cores} OpenMP threads"}
    return rec, outs


# ---------------------------------------------------------------- batched workload
def run_batch_workload(args):
    """64 seeded disks of uneven sizes (JMAX in {64,128,256}, KMAX in
    {32,64,128}, LMAX in {64,128,256}, random slope and H/r): one step = one
    replay of a CUDA graph holding chy_solve_multi over all of them; the FP64
    path is timed the same way.  One GPU (the rank-0 device)."""
    import torch
    import chymera_uo_b200 as chy
    from chymera_uo_b200 import synth
    rank, local, ws = dist_info()
    torch.cuda.set_device(local)
    n = 64
    dens = [synth.config_density(4, i) for i in range(n)]
    rhos = [chy.to_cuda_fortran(r) for r, _ in dens]
    res = {}
    for prec in ("mixed", "fp64"):
        cache = {}
        plans = []
        for _, g in dens:
            key = (g.jmax, g.kmax, g.lmax)
            if key not in cache:
                cache[key] = chy.Plan(chy.grid(*key), prec, 8)
            plans.append(cache[key])
        outs = [chy.fortran_zeros_cuda(p.shape) for p in plans]
        chy.solve_multi(plans, rhos, outs)          # side streams and smem attributes before capture
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            chy.solve_multi(plans, rhos, outs)
        for _ in range(args.warmup):
            graph.replay()
        torch.cuda.synchronize()
        launches0 = sum(p.launches for p in cache.values())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(torch.cuda.current_device()) as clk:
            e0.record()
            for _ in range(args.steps):
                graph.replay()
            e1.record()
            torch.cuda.synchronize()
        res[prec] = {"ms": e0.elapsed_time(e1), "outs": outs, "clocks": clk.summary(),
                     "sizes": len(cache), "plans": cache}
        del graph
    worst = 0.0
    for (_, g), a, b in zip(dens, res["mixed"]["outs"], res["fp64"]["outs"]):
        sl = (slice(0, g.jmax + 1), slice(0, g.kmax + 1))
        worst = max(worst, float(torch.linalg.vector_norm(a[sl] - b[sl]) / torch.linalg.vector_norm(b[sl])))
    ms = res["mixed"]["ms"]
    value = n * args.steps / (ms * 1e-3)
    line = {"metric": "pot3 solves/s, 64 uneven grids per CUDA-graph replay (mixed vs FP64)", "value": value,
            "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "mixed: f16 hi/lo tensor-core + f32 + f64", "data": "synthetic",
            "config": {"workload": "batched: 64 seeded disks, JMAX {64,128,256} x KMAX {32,64,128} x "
                                   "LMAX {64,128,256}, slope U[-2,-1], H/r U[0.03,0.1]",
                       "distinct_grids": res["mixed"]["sizes"], "solves_per_step": n,
                       "launch": "one CUDA graph replay of chy_solve_multi per step",
                       "l2": "inputs larger than L2 (all 64 densities resident)"},
            "fp64_gpu": {"value": n * args.steps / (res["fp64"]["ms"] * 1e-3), "unit": UNIT,
                         "ms_per_step": res["fp64"]["ms"] / args.steps},
            "accuracy": {"rel_l2_mixed_vs_fp64_max": worst},
            "clocks": res["mixed"]["clocks"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- time-step workload
STAR = dict(mass_star=1.0, tmassacc=0.0125, rpstar=0.0031, phi_star=0.7)


def source_bytes_per_launch(jh=J, kh=K, jmin=2):
    """Algorithmic HBM bytes of one SOURCE launch: per updated cell
    (J = JSTART..JMAX+1, K = 2..KMAX+1, every L) it reads RHO, PHI, OMEGA, P,
    S, T, A once and writes S, T, A once, 10 x 8 bytes."""
    jstart = max(jmin, 2)
    return 80 * (jh + 2 - jstart) * kh * L


def run_step_workload(args):
    """The gravity of one hydro time step at 256x128x256, in the reference's
    order (radhydro/3dhyd-main.f:474-524): BDYGEN + POT3, ExternalPot (fused
    into the inverse transform), then SOURCE's potential, pressure and
    rotation terms.  One solve per step, as the reference does; device
    arrays.  Reports steps/s, the inverse transform with and without the star
    potential, and the SOURCE kernel against the HBM roofline."""
    import torch
    import chymera_uo_b200 as chy
    rank, local, ws = dist_info()
    torch.cuda.set_device(local)
    rho = chy.to_cuda_fortran(densities(1, rank)[0])
    phi = chy.fortran_zeros_cuda((J + 2, K + 2, L))
    rng = np.random.default_rng(5 + rank)
    hyd = {k: chy.to_cuda_fortran(np.asfortranarray(rng.random((J + 2, K + 2, L)))) for k in
           ("omega", "p", "s", "t", "a")}
    g = chy.grid(J, K, L)
    plan = chy.Plan(g, args.precision, 1)
    plan.set_external(**STAR)
    bare = chy.Plan(g, args.precision, 1)
    stream = torch.cuda.current_stream()
    delt = 1e-6

    def step(p, with_source=True):
        p.solve(rho, phi)
        if with_source:
            p.source(rho, phi, hyd["omega"], hyd["p"], hyd["s"], hyd["t"], hyd["a"], delt)

    for _ in range(args.warmup):
        step(plan)
        step(bare, False)
    torch.cuda.synchronize()
    # whole steps
    launches0 = plan.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step(plan)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    gpu_launches = plan.launches - launches0
    # stage times with and without the star potential
    inv = {}
    for name, p in (("with_star", plan), ("without_star", bare)):
        p.set_profiling(True)
        for _ in range(args.steps):
            p.solve(rho, phi)
        torch.cuda.synchronize()
        st, calls = p.stage_times()
        p.set_profiling(False)
        inv[name] = st["inverse+ghosts+zaxphi"] / max(calls, 1)
    # SOURCE alone: right after a solve (PHI partly in L2) and after an L2 flush
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    src = {}
    for name, flush_first in (("after_solve", False), ("after_l2_flush", True)):
        tot = 0.0
        for _ in range(args.steps):
            plan.solve(rho, phi)
            if flush_first:
                flush.fill_(1)
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            plan.source(rho, phi, hyd["omega"], hyd["p"], hyd["s"], hyd["t"], hyd["a"], delt)
            a1.record(stream)
            torch.cuda.synchronize()
            tot += a0.elapsed_time(a1)
        src[name] = tot / args.steps
    hbm, kind = peaks()
    sb = source_bytes_per_launch()
    achieved = sb / (src["after_l2_flush"] * 1e-3) / 1e9
    line = {"metric": "gravity steps/s @256x128x256: BDYGEN+POT3, ExternalPot, SOURCE", "value":
            args.steps / (ms * 1e-3), "unit": "steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "mixed: f16 hi/lo tensor-core + f32 + f64; f64 star potential and sources"
            if args.precision == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": "one time step's gravity: seeded disk, star at (0.0031, 0.7 rad), "
                                   "random OMEGA, P, S, T, A; device arrays", "precision": args.precision,
                       "l2": "SOURCE timed after a 256 MiB L2 flush for the roofline"},
            "gpu_launches": gpu_launches,
            "inverse_ms": inv, "source_ms": src,
            "roofline_source": {"bound": "hbm", "achieved": achieved, "peak": hbm,
                                "unit": "GB/s", "frac": achieved / hbm, "peak_kind": kind,
                                "algorithmic_bytes": sb},
            "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- serving workload
def run_serving_workload(args):
    """Poisson request streams (mean rates --rates) of seeded disks with the
    serving mix of grid sizes (20% 512x128x512, the rest drawn from the batched
    size set) through chy_server; reports solves/s and p50/p99 latency per rate
    for the mixed-precision server and the plain FP64 server."""
    import threading
    import torch
    import chymera_uo_b200 as chy
    from chymera_uo_b200 import synth
    rank, local, ws = dist_info()
    torch.cuda.set_device(local)
    # a pool of distinct requests, reused round robin (a pool entry is
    # resubmitted only after its previous request finished)
    pool_n = 48
    pool = []
    for i in range(pool_n):
        rho, g = synth.config_density(5, i)
        a = chy.pinned_fortran(rho.shape)
        a[...] = rho
        f = chy.pinned_fortran(rho.shape)
        f[...] = 0.0
        pool.append(((g.jmax, g.kmax, g.lmax), a, f))
    rates = [float(r) for r in args.rates.split(",") if r]
    out = []
    for prec in ("mixed", "fp64"):
        srv = chy.Server(prec, hbm_budget=96 << 30, max_batch=4)
        grids = {k: chy.grid(*k) for k, _, _ in pool}
        # warm every size class once (plans are created on first use)
        for t in [srv.submit(grids[k], a, f) for k, a, f in pool]:
            srv.wait(t)
        for rate in rates:
            n = args.requests
            rng = np.random.default_rng(int(rate))
            gaps = rng.exponential(1.0 / rate, n)
            tickets = [None] * n
            last = [None] * pool_n
            lat = [0.0] * n
            lock = threading.Lock()

            def producer():
                t0 = time.perf_counter()
                due = t0
                for i in range(n):
                    due += gaps[i]
                    d = due - time.perf_counter()
                    if d > 0:
                        time.sleep(d)
                    j = i % pool_n
                    if last[j] is not None:
                        lat[last[j]] = srv.wait(tickets[last[j]])
                    k, a, f = pool[j]
                    with lock:
                        tickets[i] = srv.submit(grids[k], a, f)
                    last[j] = i

            st0 = srv.stats()
            t_start = time.perf_counter()
            th = threading.Thread(target=producer)
            th.start()
            th.join()
            for j in range(pool_n):
                if last[j] is not None:
                    lat[last[j]] = srv.wait(tickets[last[j]])
            wall = time.perf_counter() - t_start
            st1 = srv.stats()
            out.append({"precision": prec, "rate_req_s": rate, "requests": n, "solves_per_s": n / wall,
                        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                        "batches": st1["batches"] - st0["batches"]})
        srv.close()
    line = {"metric": "pot3 serving: solves/s and p50/p99 latency vs Poisson arrival rate (mixed vs FP64)",
            "value": max(r["solves_per_s"] for r in out if r["precision"] == "mixed"), "unit": UNIT,
            "n_gpus": ws, "higher_is_better": True, "data": "synthetic",
            "config": {"workload": "serving: seeded disks, 20% 512x128x512, 80% from the batched size set; "
                                   f"{pool_n} distinct requests reused round robin; pinned host buffers; "
                                   "latency = submit to completion on the host clock",
                       "server": "chy_server, max_batch 4, two lanes per grid"},
            "per_rate": out}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU arm
def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=32, help="solves per step (launch sequence)")
    ap.add_argument("--impl", default="chymera", choices=["chymera", "reference"])
    ap.add_argument("--refine", type=int, default=1, help="mixed-precision refinement corrections")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="mode-solve path of the timed plan (fp64: the plain FP64 GPU path)")
    ap.add_argument("--latency-samples", type=int, default=200)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="pot3", choices=["pot3", "batch", "serving", "step"],
                    help="pot3: 256x128x256 mixed (default); batch: 64 uneven grids from one captured "
                         "graph; serving: Poisson request stream with p50/p99 latency; step: one time "
                         "step's gravity (solve, star potential, SOURCE terms)")
    ap.add_argument("--rates", default="200,1000,5000", help="serving: mean arrival rates (req/s)")
    ap.add_argument("--requests", type=int, default=400, help="serving: requests per rate")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch_workload(args)
    if args.workload == "serving":
        return run_serving_workload(args)
    if args.workload == "step":
        return run_step_workload(args)

    import torch
    import chymera_uo_b200 as chy

    rank, local, ws = dist_info()
    torch.cuda.set_device(local)
    dist = init_replicas(ws, local)

    def barrier():
        replica_barrier(dist, "cuda")

    def max_over_ranks(x):
        return replica_max(dist, x, "cuda")

    B = args.batch
    host = densities(B, rank * B)
    rhos = [chy.to_cuda_fortran(r) for r in host]
    phis = [chy.fortran_zeros_cuda((J + 2, K + 2, L)) for _ in range(B)]
    ref_phis = [chy.fortran_zeros_cuda((J + 2, K + 2, L)) for _ in range(B)]
    g = chy.grid(J, K, L)
    plan = chy.Plan(g, args.precision, B)
    if args.precision == "mixed":
        plan.set_refine(args.refine)
    plan64 = chy.Plan(g, "fp64", B)
    stream = torch.cuda.current_stream()

    # ---- device-resident throughput (the `value`)
    for _ in range(args.warmup):
        plan.solve_batch(rhos, phis)
    barrier()
    plan.set_profiling(True)
    launches0 = plan.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            plan.solve_batch(rhos, phis)
        e1.record(stream)
        barrier()
    gpu_launches = plan.launches - launches0
    ms = max_over_ranks(e0.elapsed_time(e1))
    stage, calls = plan.stage_times()
    plan.set_profiling(False)
    clocks = clk.summary()
    value = replica_value(ws, B, args.steps, ms)

    # ---- dominant kernel: the mode solves (one launch per step)
    mode_ms = stage["mode solves"] / max(calls, 1)
    alg = mode_solve_bytes_per_solve() * B
    hbm, peak_kind = peaks()
    achieved = alg / (mode_ms * 1e-3) / 1e9
    tps = profiled_traffic_per_solve() if args.precision == "mixed" else None
    kname = "k_mode_mixed" if args.precision == "mixed" else "FP64 mode solves (k_zfwd_f64, k_thomas_f64, k_zinv_f64)"
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_kind": f"{peak_kind} (MEASURED_PEAKS hbm_gbs)",
                "traffic": None if tps is None else tps * B,
                "algorithmic_bytes": alg, "launch_ms": mode_ms,
                "stage_ms_per_step": {k: v / max(calls, 1) for k, v in stage.items()}}

    # ---- plain FP64 GPU path on the same inputs (same step shape)
    for _ in range(args.warmup):
        plan64.solve_batch(rhos, ref_phis)
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k64 = max(3, args.steps // 2)
    f0.record(stream)
    for _ in range(k64):
        plan64.solve_batch(rhos, ref_phis)
    f1.record(stream)
    barrier()
    ms64 = max_over_ranks(f0.elapsed_time(f1))
    fp64_value = ws * B * k64 / (ms64 * 1e-3)

    # ---- accuracy: mixed vs the FP64 GPU path, device status words
    _, diags = plan.solve_batch(rhos, phis, diag=True)
    torch.cuda.synchronize()
    errs, maxe = [], []
    for a, b in zip(phis, ref_phis):
        d = (a[: J + 1, : K + 1] - b[: J + 1, : K + 1])
        errs.append(float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(b[: J + 1, : K + 1])))
        maxe.append(float(d.abs().max() / b[: J + 1, : K + 1].abs().max()))
    accuracy = {"rel_l2_vs_fp64_gpu_max": max(errs), "max_rel_vs_fp64_gpu": max(maxe),
                "corr_rel_solve0": diags[0]["corr_rel"], "solves_checked": B}

    # ---- single-solve latency (device-resident, one launch sequence each)
    lat = []
    one_r, one_p = rhos[:1], phis[:1]
    for _ in range(3):
        plan.solve_batch(one_r, one_p)
    barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.latency_samples)]
    for i in range(args.latency_samples):
        evs[i][0].record(stream)
        plan.solve_batch([rhos[i % B]], [phis[i % B]])
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    lat = [a.elapsed_time(b) for a, b in evs]
    latency = {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
               "samples": len(lat), "what": "device time of one solve (batch 1), inputs in HBM"}

    # ---- end to end through the public API: pinned host RHO in, PHI out
    pin_r = [torch.empty((L, K + 2, J + 2), dtype=torch.float64, pin_memory=True).numpy().transpose()
             for _ in range(B)]
    pin_p = [torch.empty((L, K + 2, J + 2), dtype=torch.float64, pin_memory=True).numpy().transpose()
             for _ in range(B)]
    for a, b in zip(pin_r, host):
        a[...] = b
    for a in pin_p:
        a[...] = 0.0
    h2d = B * 8 * (J + 2) * (K + 2) * L                      # RHO
    d2h = B * 8 * L * (K * (J + 2) + (J + 1))                # PHI's write set
    ke = max(3, args.steps // 4)
    for _ in range(args.warmup):
        plan.solve_batch(pin_r, pin_p)
    barrier()
    dstream = torch.cuda.default_stream()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(dstream)
    for _ in range(ke):
        plan.solve_batch(pin_r, pin_p)
    h1.record(dstream)
    barrier()
    mse = max_over_ranks(h0.elapsed_time(h1))
    e2e = {"value": ws * B * ke / (mse * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "steps": ke,
           "api": "chy_solve_batch with CHY_PTR_HOST (pinned numpy buffers)"}
    host_ok = np.array_equal(pin_p[0], phis[0].cpu().numpy())
    accuracy["host_path_equals_device_path"] = bool(host_ok)

    # ---- CPU baseline (oracle port), rank 0 at N=1 only; also checks results
    cpu = None
    if ws == 1 and rank == 0 and not args.no_cpu_baseline:
        cpu, outs = cpu_baseline(host, args.cpu_seconds, 8)
        ws_sl = (slice(0, J + 1), slice(0, K + 1))
        got = [p.cpu().numpy() for p in phis[: len(outs)]]
        g64 = [p.cpu().numpy() for p in ref_phis[: len(outs)]]
        accuracy["rel_l2_mixed_vs_oracle_max"] = max(rel_l2(a[ws_sl], b[ws_sl]) for a, b in zip(got, outs))
        accuracy["rel_l2_fp64_vs_oracle_max"] = max(rel_l2(a[ws_sl], b[ws_sl]) for a, b in zip(g64, outs))
        accuracy["oracle_solves_compared"] = len(outs)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "mixed: f16 hi/lo tensor-core + f32 + f64" if args.precision == "mixed" else "f64",
                "data": "synthetic",
                "config": {"workload": WORKLOAD if args.precision == "mixed" else
                           WORKLOAD.replace("mixed precision", "plain FP64 GPU path"), "jmax": J, "kmax": K, "lmax": L, "solves_per_step": B,
                           "refine_corrections": args.refine, "parallelism": f"replicas x{ws}",
                           "l2": f"inputs larger than L2 ({B} x {8 * (J + 2) * (K + 2) * L / 1e6:.0f} MB "
                                 "RHO + PHI resident)"},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": gpu_launches,
                "clocks": clocks, "latency_ms": latency,
                "fp64_gpu": {"value": fp64_value, "unit": UNIT, "ms_per_step": ms64 / k64,
                             "mixed_over_fp64": value / fp64_value},
                "accuracy": accuracy}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
