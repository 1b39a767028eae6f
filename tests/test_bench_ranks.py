"""`bench.py --gpus N` starts its own N ranks when no launcher did.

Run on CPU with the host-only chain workload: the spawner runs torchrun
with two local ranks over gloo, each rank takes its own sample columns,
and rank 0 prints one line with n_gpus = 2 and the moments averaged over
all ranks' columns, equal to the single-process computation over the same
global columns.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_spawns_ranks_and_combines_their_moments():
    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    env["CUDA_VISIBLE_DEVICES"] = ""
    env["OMP_NUM_THREADS"] = "1"
    out = subprocess.run([sys.executable, "bench.py", "--workload", "chain", "--gpus", "2",
                          "--steps", "2", "--warmup", "1"], cwd=ROOT, env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    line = lines[0]
    assert line["n_gpus"] == 2
    sys.path.insert(0, ROOT)
    import bench
    want = bench.chain_moments(4096, 0, 8, 64) / 8
    assert np.abs(np.array(line["moments"]) - want).max() < 1e-12
