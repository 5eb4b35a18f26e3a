"""The multi-GPU bench runs replicas: each rank solves its own densities and the
only collectives are the barrier around the timed region and the max of the
ranks' times.  Checked here with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    import bench
    dist = bench.init_replicas(ws, rank, backend="gloo", timeout_s=30)
    bench.replica_barrier(dist, "cpu")
    ms = 100.0 + 50.0 * rank                   # rank 1 is the slowest
    ms_max = bench.replica_max(dist, ms, "cpu")
    out[rank] = (ms_max, bench.replica_value(ws, 32, 10, ms_max))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_takes_the_slowest_rank():
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        assert out[0] == out[1]
        ms_max, value = out[0]
    assert ms_max == 150.0
    assert value == pytest.approx(2 * 32 * 10 / 0.150)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import sys
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        steps, warmup = 1, 3
    assert bench.run_reference(Args()) == 0
    assert capsys.readouterr().out == ""
