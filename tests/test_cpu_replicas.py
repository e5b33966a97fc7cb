"""Multi-GPU runs are replicas (the path does not shard): the bench's
barrier and max-over-ranks on world_size 2 with gloo on the CPU, the
whole-job rate, and the reference arm under torchrun printing one line from
rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist(world, rank, backend="gloo")
    try:
        d.barrier()
        out[rank] = d.max(10.0 + rank)   # rank 1 is the slowest
        d.barrier()
    finally:
        d.close()


def test_dist_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp   # imported here, not at collection time
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        assert dict(out) == {0: 11.0, 1: 11.0}


def test_aggregate_rate_is_weak_scaling():
    sys.path.insert(0, ROOT)
    import bench
    one = bench.aggregate_rate(1e8, 10, 1, 500.0)
    assert one == pytest.approx(2e9)
    # two replicas in the time of the slower one: twice the units
    assert bench.aggregate_rate(1e8, 10, 2, 500.0) == pytest.approx(2 * one)


def test_reference_arm_under_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--ref-budget", "0.1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_line_at_one_process():
    """The reference arm's line carries the contract's keys, on the metric,
    unit and workload the GPU arm reports (the module's shared constants)."""
    import bench
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0",
           "--ref-budget", "0.1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e", "impl"):
        assert k in d, k
    assert (d["metric"], d["unit"], d["config"]["workload"]) == (bench.METRIC, bench.UNIT, bench.WORKLOAD_NAME)
    assert d["impl"] == "reference" and d["n_gpus"] == 1 and d["steps"] == 1 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
