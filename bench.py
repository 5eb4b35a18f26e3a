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


def profiled_traffic_per_solve(kernel: str = "k_mode_pair"):
    """DRAM bytes (read + write) per solve of the mode-solve kernel from the
    committed ncu summary of that kernel, or None."""
    path = os.path.join(HERE, "profiles", f"{kernel}_256x128x256.md")
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
def batched_record(steps, warmup, precisions=("mixed", "fp64", "blktri")):
    """64 seeded disks of uneven sizes (JMAX in {64,128,256}, KMAX in
    {32,64,128}, LMAX in {64,128,256}, random slope and H/r): one step = one
    replay of a CUDA graph holding chy_solve_multi over all of them, for each
    mode-solve path.  Returns the record (device times, CUDA events)."""
    import torch
    import chymera_uo_b200 as chy
    from chymera_uo_b200 import synth
    n = 64
    dens = [synth.config_density(4, i) for i in range(n)]
    rhos = [chy.to_cuda_fortran(r) for r, _ in dens]
    res = {}
    for prec in precisions:
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
        # the launch schedule of this request set, picked by timing (kept in the plans)
        tune = chy.autotune_multi(plans, rhos, outs, repeats=2 if prec == "blktri" else 3)
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            chy.solve_multi(plans, rhos, outs)
        for _ in range(warmup):
            graph.replay()
        torch.cuda.synchronize()
        k = steps if prec != "blktri" else max(3, steps // 4)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(torch.cuda.current_device()) as clk:
            e0.record()
            for _ in range(k):
                graph.replay()
            e1.record()
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / k
        res[prec] = {"ms": ms, "outs": outs, "clocks": clk.summary(), "sizes": len(cache),
                     "value": n / (ms * 1e-3), "steps": k, "tune": tune}
        del graph, cache, plans
    worst = {}
    base = "blktri" if "blktri" in res else "fp64"
    for prec in res:
        if prec == base:
            continue
        w = 0.0
        for (_, g), a, b in zip(dens, res[prec]["outs"], res[base]["outs"]):
            sl = (slice(0, g.jmax + 1), slice(0, g.kmax + 1))
            w = max(w, float(torch.linalg.vector_norm(a[sl] - b[sl]) / torch.linalg.vector_norm(b[sl])))
        worst[f"rel_l2_{prec}_vs_{base}_max"] = w
    rec = {"metric": "pot3 solves/s, 64 uneven grids per CUDA-graph replay", "unit": UNIT,
           "value": res["mixed"]["value"] if "mixed" in res else None,
           "per_precision": {p: {"value": r["value"], "ms_per_step": r["ms"], "steps": r["steps"],
                                 "schedule": r["tune"]}
                             for p, r in res.items()},
           "config": {"workload": "batched: 64 seeded disks, JMAX {64,128,256} x KMAX {32,64,128} x "
                                  "LMAX {64,128,256}, slope U[-2,-1], H/r U[0.03,0.1]",
                      "distinct_grids": next(iter(res.values()))["sizes"], "solves_per_step": n,
                      "launch": "one CUDA graph replay of chy_solve_multi per step (grids on side streams), "
                                "schedule picked by chy_autotune_multi before capture (schedule.ms_default: "
                                "the default schedule's time per call, outside the graph)",
                      "l2": "inputs larger than L2 (all 64 densities resident)"},
           "accuracy": worst, "clocks": res[precisions[0]]["clocks"]}
    for p in res:
        if p != "mixed" and "mixed" in res:
            rec[f"mixed_over_{p}"] = res["mixed"]["value"] / res[p]["value"]
    return rec


def run_batch_workload(args):
    """The batched workload alone (one GPU, the rank-0 device)."""
    import torch
    rank, local, ws = dist_info()
    torch.cuda.set_device(local)
    rec = batched_record(args.steps, args.warmup)
    line = {"metric": rec["metric"] + " (mixed vs FP64)", "value": rec["value"], "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": rec["per_precision"]["mixed"]["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "mixed: f16 hi/lo tensor-core + f32 + f64", "data": "synthetic", "config": rec["config"],
            "per_precision": rec["per_precision"], "accuracy": rec["accuracy"], "clocks": rec["clocks"]}
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
def serving_record(rates, max_requests, seconds_per_rate, precisions=("mixed", "fp64")):
    """Poisson request streams at each mean rate in `rates` of seeded disks
    with the serving mix of grid sizes (20% 512x128x512, the rest drawn from
    the batched size set) through chy_server: min(max_requests, rate x
    seconds_per_rate) requests per rate.  Reports solves/s and p50/p99
    latency per rate for each precision."""
    import threading
    import chymera_uo_b200 as chy
    from chymera_uo_b200 import synth
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
    big = sum(1 for k, _, _ in pool if k == (512, 128, 512))
    out = []
    for prec in precisions:
        srv = chy.Server(prec, hbm_budget=96 << 30, max_batch=4)
        grids = {k: chy.grid(*k) for k, _, _ in pool}
        # warm every size class once (plans are created on first use)
        for t in [srv.submit(grids[k], a, f) for k, a, f in pool]:
            srv.wait(t)
        for rate in rates:
            n = int(min(max_requests, max(pool_n, round(rate * seconds_per_rate))))
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
            out.append({"precision": prec, "rate_req_s": rate, "requests": n, "wall_s": wall,
                        "solves_per_s": n / wall, "p50_ms": float(np.percentile(lat, 50)),
                        "p99_ms": float(np.percentile(lat, 99)), "batches": st1["batches"] - st0["batches"]})
        srv.close()
    return {"metric": "pot3 serving: solves/s and p50/p99 latency vs Poisson arrival rate", "unit": UNIT,
            "value": max(r["solves_per_s"] for r in out if r["precision"] == precisions[0]),
            "config": {"workload": f"serving: seeded disks, 20% 512x128x512 ({big} of {pool_n} pool entries), "
                                   "80% from the batched size set; min(10000, rate x "
                                   f"{seconds_per_rate:g} s) requests per rate; {pool_n} distinct requests "
                                   "reused round robin; pinned host buffers; latency = submit to completion "
                                   "on the host clock",
                       "server": "chy_server, max_batch 4, two lanes per grid",
                       "precisions": list(precisions)},
            "per_rate": out}


def run_serving_workload(args):
    """The serving workload alone (one GPU, the rank-0 device)."""
    import torch
    rank, local, ws = dist_info()
    torch.cuda.set_device(local)
    rates = [float(r) for r in args.rates.split(",") if r]
    rec = serving_record(rates, args.requests, args.serve_seconds)
    line = {"metric": rec["metric"] + " (mixed vs FP64)", "value": rec["value"], "unit": UNIT, "n_gpus": ws,
            "higher_is_better": True, "data": "synthetic", "config": rec["config"], "per_rate": rec["per_rate"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU arm
def pcie_ceiling(nbytes=512 << 20, reps=5):
    """Pinned host <-> device copy bandwidth of this box (GB/s, CUDA events):
    each direction alone and both at once on two streams."""
    import torch
    h_in = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    h_out = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d_in = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    d_out = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def timed(fn, stream):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        return e0, e1

    with torch.cuda.stream(s1):
        d_in.copy_(h_in, non_blocking=True)
        h_out.copy_(d_out, non_blocking=True)
    torch.cuda.synchronize()
    with torch.cuda.stream(s1):
        a = timed(lambda: d_in.copy_(h_in, non_blocking=True), s1)
    torch.cuda.synchronize()
    with torch.cuda.stream(s1):
        b = timed(lambda: h_out.copy_(d_out, non_blocking=True), s1)
    torch.cuda.synchronize()
    with torch.cuda.stream(s1):
        c = timed(lambda: d_in.copy_(h_in, non_blocking=True), s1)
    with torch.cuda.stream(s2):
        d = timed(lambda: h_out.copy_(d_out, non_blocking=True), s2)
    torch.cuda.synchronize()
    gbs = lambda ev: reps * nbytes / (ev[0].elapsed_time(ev[1]) * 1e-3) / 1e9
    return {"h2d": gbs(a), "d2h": gbs(b), "concurrent_h2d": gbs(c), "concurrent_d2h": gbs(d),
            "bytes_per_copy": nbytes}


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
    ap.add_argument("--grid", default=None,
                    help="pot3 workload: JMAX,KMAX,LMAX of the timed solves (default 256,128,256; other "
                         "grids are for profiling runs, not the metric)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64", "blktri"],
                    help="mode-solve path of the timed plan (fp64: the plain FP64 GPU path)")
    ap.add_argument("--latency-samples", type=int, default=200)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="pot3", choices=["pot3", "batch", "serving", "step"],
                    help="pot3: 256x128x256 mixed (default); batch: 64 uneven grids from one captured "
                         "graph; serving: Poisson request stream with p50/p99 latency; step: one time "
                         "step's gravity (solve, star potential, SOURCE terms)")
    ap.add_argument("--rates", default="100,300,1000,3000,5000", help="serving: mean arrival rates (req/s)")
    ap.add_argument("--requests", type=int, default=10000, help="serving: most requests per rate")
    ap.add_argument("--serve-seconds", type=float, default=10.0,
                    help="serving: requests per rate are min(--requests, rate x this)")
    ap.add_argument("--no-extra", action="store_true",
                    help="pot3 workload: skip the batched and serving records appended after the timed region")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.grid:
        global J, K, L
        J, K, L = (int(v) for v in args.grid.split(","))
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
    plan64 = chy.Plan(g, "fp64", B)          # FP64 eigenbasis mode solve
    planbk = chy.Plan(g, "blktri", B)        # FP64 in BLKTRI's order: the plain FP64 pot3
    eig_phis = [chy.fortran_zeros_cuda((J + 2, K + 2, L)) for _ in range(B)]
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
    mk = chy.lib().chy_dbg_mixed_kernel(plan._p)
    tps = profiled_traffic_per_solve({1: "k_mode_mixed", 2: "k_mode_pair"}.get(mk, "none")) \
        if args.precision == "mixed" and (J, K, L) == (256, 128, 256) else None
    mixed_kernel = {1: "k_mode_mixed", 2: "k_mode_pair (CTA pairs, two modes per SM)",
                    3: "wide mixed pipeline (k_wide_*)"}.get(mk, "mixed")
    kname = {"mixed": mixed_kernel,
             "fp64": "FP64 mode solves (k_zfwd_f64, k_thomas_f64, k_zinv_f64)",
             "blktri": "BLKTRI-order mode solves (k_blk_gather, k_blk_solve, k_blk_scatter)"}[args.precision]
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_kind": f"{peak_kind} (MEASURED_PEAKS hbm_gbs)",
                "traffic": None if tps is None else tps * B,
                "algorithmic_bytes": alg, "launch_ms": mode_ms,
                "stage_ms_per_step": {k: v / max(calls, 1) for k, v in stage.items()}}

    # ---- the FP64 GPU paths on the same inputs (same step shape): BLKTRI's
    # order (the plain FP64 pot3, the reference's rounding) and the eigenbasis
    def time_path(pl, outs, k):
        for _ in range(args.warmup):
            pl.solve_batch(rhos, outs)
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(k):
            pl.solve_batch(rhos, outs)
        f1.record(stream)
        barrier()
        m = max_over_ranks(f0.elapsed_time(f1))
        return ws * B * k / (m * 1e-3), m / k, k

    bk_value, bk_ms, bk_k = time_path(planbk, ref_phis, 3)
    eig_value, eig_ms, eig_k = time_path(plan64, eig_phis, max(3, args.steps // 2))

    # ---- accuracy: mixed and the eigenbasis path vs the BLKTRI-order FP64
    # path, device status words
    _, diags = plan.solve_batch(rhos, phis, diag=True)
    torch.cuda.synchronize()

    def worst(xs, ys):
        errs, maxe = [], []
        for a, b in zip(xs, ys):
            d = (a[: J + 1, : K + 1] - b[: J + 1, : K + 1])
            errs.append(float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(b[: J + 1, : K + 1])))
            maxe.append(float(d.abs().max() / b[: J + 1, : K + 1].abs().max()))
        return max(errs), max(maxe)

    e_mx, m_mx = worst(phis, ref_phis)
    e_eg, _ = worst(eig_phis, ref_phis)
    accuracy = {"rel_l2_vs_fp64_gpu_max": e_mx, "max_rel_vs_fp64_gpu": m_mx,
                "fp64_gpu_reference": "BLKTRI-order FP64 path (CHY_PREC_FP64_BLKTRI)",
                "rel_l2_fp64_eigen_vs_blktri_max": e_eg,
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
    # the library's copies per solve: RHO whole and PHI's untouched cells in,
    # PHI whole out (chymera_uo_b200/csrc/planimpl.h)
    vol = (J + 2) * (K + 2) * L
    h2d = B * 8 * (vol + L * (J + 3))
    d2h = B * 8 * vol
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
    pcie = pcie_ceiling()
    e2e["pcie_gbs"] = pcie
    e2e["achieved_gbs"] = {"h2d": h2d * ke / (mse * 1e-3) / 1e9, "d2h": d2h * ke / (mse * 1e-3) / 1e9}
    e2e["pcie_frac"] = max(e2e["achieved_gbs"]["h2d"] / pcie["concurrent_h2d"],
                           e2e["achieved_gbs"]["d2h"] / pcie["concurrent_d2h"])
    host_ok = np.array_equal(pin_p[0], phis[0].cpu().numpy())
    accuracy["host_path_equals_device_path"] = bool(host_ok)

    # ---- CPU baseline (oracle port), rank 0 at N=1 only; also checks results
    cpu = None
    if ws == 1 and rank == 0 and not args.no_cpu_baseline:
        cpu, outs = cpu_baseline(host, args.cpu_seconds, 8)
        ws_sl = (slice(0, J + 1), slice(0, K + 1))
        got = [p.cpu().numpy() for p in phis[: len(outs)]]
        g64 = [p.cpu().numpy() for p in ref_phis[: len(outs)]]
        geg = [p.cpu().numpy() for p in eig_phis[: len(outs)]]
        accuracy["rel_l2_mixed_vs_oracle_max"] = max(rel_l2(a[ws_sl], b[ws_sl]) for a, b in zip(got, outs))
        accuracy["rel_l2_fp64_vs_oracle_max"] = max(rel_l2(a[ws_sl], b[ws_sl]) for a, b in zip(g64, outs))
        accuracy["rel_l2_fp64_eigen_vs_oracle_max"] = max(rel_l2(a[ws_sl], b[ws_sl]) for a, b in zip(geg, outs))
        accuracy["oracle_solves_compared"] = len(outs)
        if args.precision == "mixed":
            # the error against the oracle after each refinement step: 0 = the
            # first approximate solve alone, 1 = one FP64 correction (the
            # default), 2 = two
            per_step = {}
            nr = min(2, len(outs))
            for r in (0, 1, 2):
                pr = chy.Plan(chy.grid(J, K, L), "mixed", nr)
                pr.set_refine(r)
                o = [chy.fortran_zeros_cuda(p.shape) for p in phis[:nr]]
                pr.solve_batch(rhos[:nr], o)
                torch.cuda.synchronize()
                per_step[str(r)] = max(rel_l2(a.cpu().numpy()[ws_sl], b[ws_sl]) for a, b in zip(o, outs[:nr]))
                pr.close()
            accuracy["rel_l2_mixed_vs_oracle_per_refinement"] = per_step

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
                "fp64_gpu": {"value": bk_value, "unit": UNIT, "ms_per_step": bk_ms, "steps": bk_k,
                             "path": "plain FP64 pot3: BLKTRI generalized cyclic reduction in the "
                                     "reference's order (CHY_PREC_FP64_BLKTRI)",
                             "mixed_over_fp64": value / bk_value,
                             "eigen": {"value": eig_value, "unit": UNIT, "ms_per_step": eig_ms, "steps": eig_k,
                                       "path": "FP64 eigenbasis + radial Thomas (CHY_PREC_FP64)",
                                       "mixed_over_eigen": value / eig_value}},
                "accuracy": accuracy}
        if ws == 1 and not args.no_extra:
            # configs 4 and 5, after the timed region
            del plan64, planbk
            torch.cuda.empty_cache()
            line["batched"] = batched_record(5, 3)
            line["serving"] = serving_record([float(r) for r in args.rates.split(",") if r], args.requests,
                                             args.serve_seconds)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
