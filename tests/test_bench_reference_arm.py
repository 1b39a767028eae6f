"""The reference arm of bench.py runs on the host only.

`bench.py --impl reference` times the oracle's FP64 restatement of the KPM
recurrence (the reference itself cannot be built here).  Its operator, its
graph-local S^-1/2 factor (the reference's eigen route) and its spectral
window are built with numpy and the oracle, so the timed CPU path never
loads the CUDA library: the process must not import the library's binding
module, and the line must name the same workload config as the GPU arm's.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_never_loads_the_cuda_library():
    code = (
        "import sys, runpy\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--small', '--steps', '1', "
        "'--warmup', '0']\n"
        "runpy.run_path('bench.py', run_name='__main__')\n"
        "bad = [m for m in ('rsatb_b200._capi', 'rsatb_b200.vbcsr', 'rsatb_b200.isqrt', "
        "'rsatb_b200.calc') if m in sys.modules]\n"
        "print('IMPORTED', bad)\n")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    assert lines[-1] == "IMPORTED []", lines[-1]
    line = json.loads(lines[-2])
    assert line["impl"] == "reference"
    assert line["cuda_library_loaded"] is False
    assert line["cpu_baseline"]["kind"] == "port"
    assert line["cpu_baseline"]["sample"].startswith("8 moments")
    cfg = line["config"]
    assert cfg["n_rows"] == 13824 and cfg["vectors_per_gpu"] == 32 and cfg["block_size"] == 8
    assert "bounds_ev" not in cfg and "parallelism" not in cfg


def test_host_factor_equals_the_eigen_route():
    """oracle.graph_inverse_sqrt_eigen (batched, process pool) against the
    one-problem-at-a-time clamped eigen action on a small diamond S."""
    import numpy as np
    import oracle
    from rsatb_b200 import lattice
    _, S = lattice.diamond_lcao(L=2, seed=3)
    Z = oracle.graph_inverse_sqrt_eigen(S.row_ptr, S.col_ind, S.values, 8, workers=2, chunk=16)
    members, slot, gather = lattice.subgraph_problems(S)
    n, k = members.shape
    for i in (0, 5, n - 1):
        M = np.zeros((k * 8, k * 8))
        for p in range(k):
            for q in range(k):
                if gather[i, p, q] >= 0:
                    M[p * 8:(p + 1) * 8, q * 8:(q + 1) * 8] = S.values[gather[i, p, q]]
        X = oracle.isqrt_columns_eigen(M, slot[i] * 8, 8).T  # rows of M^-1/2 at i
        for p in range(k):
            assert np.abs(Z[i * k + p] - X[:, p * 8:(p + 1) * 8]).max() < 1e-12
