"""bench.py on N > 1 ranks (replicas, one process per GPU): the host-side aggregation, run as
world-size-2 gloo process groups on the CPU.  The slowest rank's time is the job's time, every
rank sees the same number, and the reference arm runs on rank 0 only."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, out):
    import torch.distributed as dist
    from datetime import timedelta
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(times[rank], world, "cpu")
        out[rank] = ms
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("times", [(1.25, 0.75), (0.5, 2.0)])
def test_max_over_ranks_gloo(times):
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, port, list(times), out), nprocs=world,
                       join=True, start_method="spawn")
    assert out[0] == out[1] == max(times)
    # whole-job throughput of N replicas over the slowest rank's time
    assert world * 1000.0 / out[0] == pytest.approx(world * 1000.0 / max(times))


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5


def test_reference_arm_runs_on_rank_zero_only():
    import bench
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(None, rank=1, world=2)  # a non-zero rank does no work
    assert buf.getvalue() == ""


def test_trace_bytes():
    import bench
    # state + 7 steps of (λ, err, cos, kind, distinct) + 8 clock stamps + status
    assert bench.trace_d2h_bytes(7) == 56 + 7 * 32 + 64 + 4


def test_reference_arm_json_line():
    """`bench.py --impl reference` (the host-core arm) prints one JSON line with the contract's
    keys, on a small matrix so that it runs in seconds on the CPU."""
    import json
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    r = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference", "--m", "256",
                        "--n", "1024", "--steps", "2", "--warmup", "1"],
                       capture_output=True, text=True, timeout=300, cwd=str(root))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 2
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
