"""Multi-process paths of the benchmark on CPU (gloo, world size 2).

The tracer's work shards as replicas (every rank renders its own copy of the
view; the path has no data exchange), so the only cross-rank steps are the
barrier and the max of the per-rank times.  These tests run them as two gloo
ranks on 127.0.0.1, and run the reference arm under torchrun with two ranks:
rank 0 prints the one JSON line, rank 1 exits without work."""
import json
import os
import socket
import subprocess
import sys
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    r, w, local, dist = bench.init_ranks()
    assert (r, w, local) == (rank, world, rank) and dist is not None
    slowest = bench.max_over_ranks(dist, 10.0 + 5.0 * rank)   # per-rank step times 10 and 15 ms
    dist.barrier()
    value = bench.whole_job_mrays(w, 1000, slowest * 1e-3)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as fh:
        json.dump({"slowest": slowest, "value": value}, fh)
    dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value():
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(2, _free_port(), d), nprocs=2, join=True, start_method="spawn")
        res = [json.load(open(os.path.join(d, f"rank{r}.json"))) for r in range(2)]
    assert res[0] == res[1]
    assert res[0]["slowest"] == 15.0
    # 2 ranks x 1000 rays in the slowest rank's 15 ms
    assert abs(res[0]["value"] - 2 * 1000 / 0.015 / 1e6) < 1e-12


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 3.5) == 3.5


def test_reference_arm_under_torchrun_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "3", "--workload", "small-256", "--ref-step-budget", "0.2"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
