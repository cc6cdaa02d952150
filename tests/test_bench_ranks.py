"""The replicas bench's multi-rank host logic, two gloo ranks on CPU (bench.py --dry-run):
rendezvous on 127.0.0.1, a different seeded workload per rank, the max of the ranks'
step times and one JSON line from rank 0."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_replicas_take_the_max_time_and_print_once():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(_port()), "bench.py", "--gpus", "2", "--steps", "3", "--warmup", "1", "--dry-run"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    res = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, res.stdout
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["scaling"] == "weak"
    # rank 1's stand-in time (2 x 10 ms per step) is the max; value counts both ranks' paths
    assert d["ms_per_step"] == 20.0
    assert abs(d["value"] - 2 * 3 * 256 * 256 * 16 / 0.060) < 1e-6 * d["value"]
    a, b = d["rank_workload_digests"]
    assert a != b
