#!/usr/bin/env python
"""Benchmark of the KPM DOS hot path on B200: vector-moments/s of the
rescaled Chebyshev recurrence, mixed precision (FP32 matrices/vectors, FP64
rescale and moment dots) against plain FP64, on the non-orthogonal LCAO
diamond workload (N = 262,144, 8x8 BSR, sandwich Z^H H Z, R = 128
Rademacher vectors, 1024 moments).

One step = one full moment recurrence (1024 moments, 512 sandwich
applications = 1536 SpMMs) over the R sample vectors, inputs resident in
HBM; every panel (134-268 MB) is larger than the 126 MB L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (one rank per GPU; started without a launcher, bench.py runs
itself under torch.distributed.run with N local ranks) each rank runs its
own 128 sample columns (global columns rank*128 ...), the moments are summed
with one NCCL all-reduce, and the time is the max over ranks.  Prints one
JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from datetime import timedelta
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
METRIC = "KPM moments/sec & BSR SpMM HBM GB/s: mixed-prec vs FP64, at DOS err ≤1e-5"
UNIT = "vector-moments/s"
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["diamond", "graphene", "isqrt", "transport", "adjoint",
                                          "chain"],
                   default="diamond")
    p.add_argument("--si-L", type=int, default=8, help="silicon conventional cells per side")
    p.add_argument("--tbg-m", type=int, default=31, help="moire index of the TBG cell")
    p.add_argument("--tbg-tiles", type=int, default=4, help="TBG cells per side")
    p.add_argument("--transport-moments", type=int, default=2048)
    p.add_argument("--transport-samples", type=int, default=16, help="samples over all GPUs")
    p.add_argument("--isqrt-n", type=int, default=100_000,
                   help="problems of the batched inverse-sqrt workload")
    p.add_argument("--isqrt-precision", choices=["tf32x3", "tf32", "fp64"], default="tf32x3")
    p.add_argument("--isqrt-family", choices=["continuous", "gapped"], default="continuous",
                   help="spectrum family of the batched inverse-sqrt problems")
    p.add_argument("--isqrt-ws-gb", type=float, default=24.0,
                   help="device workspace per chunk of the batched inverse sqrt")
    p.add_argument("--small", action="store_true", help="reduced sizes, for a quick check")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-moments", type=int, default=8,
                   help="moments in the bounded CPU baseline sample")
    p.add_argument("--spmm-only", action="store_true",
                   help="time Y = H X alone on a diamond L^3 H (the ncu profiling case)")
    p.add_argument("--isqrt-no-autotune", action="store_true",
                   help="batched S^-1/2: built-in tensor-core tiles instead of autotuned ones")
    p.add_argument("--forms-only", action="store_true",
                   help="time one application of the sandwich and the solve forms")
    p.add_argument("--forms-L", type=int, default=8)
    p.add_argument("--spmm-L", type=int, default=12)
    p.add_argument("--spmm-reps", type=int, default=3)
    p.add_argument("--spmm-kernels", default="",
                   help="comma list of FP32 step kernels to A/B in --spmm-only (bulk, tf32, "
                        "tf32:p3, v1, ...), each with its max error against the FP64 SpMM")
    p.add_argument("--spmm-widths", default="128,32,16,8",
                   help="panel widths R of --spmm-only")
    return p.parse_args()


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if self.proc is None or not self.path:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[4:]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for name, flag in zip(names, r[3][1:]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        loaded = [r for r in rows if r[2] > 200.0] or rows
        return {"sm_mhz": statistics.median(r[0] for r in loaded),
                "sm_max_mhz": max(r[1] for r in rows),
                "power_w_max": max(r[2] for r in rows),
                "samples": len(rows), "reasons": sorted(reasons)}


# -------------------------------------------------------------- distributed

class Dist:
    """One rank per GPU (NCCL); without a GPU (the host-only chain
    workload) the ranks talk over gloo."""

    def __init__(self):
        import torch
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.torch = torch
        self.cuda = torch.cuda.is_available()
        if self.cuda:
            torch.cuda.set_device(self.local_rank)
        if self.world > 1:
            import torch.distributed as dist
            if self.cuda:
                dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                        device_id=torch.device("cuda", self.local_rank))
            else:
                dist.init_process_group("gloo", timeout=timedelta(seconds=120))
            self.dist = dist
        else:
            self.dist = None

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if self.dist is None:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64,
                              device="cuda" if self.cuda else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum_array(self, a: np.ndarray) -> np.ndarray:
        if self.dist is None:
            return a
        t = self.torch.as_tensor(np.ascontiguousarray(a))
        if self.cuda:
            t = t.cuda()
        self.dist.all_reduce(t)
        return t.cpu().numpy()

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except json.JSONDecodeError:
            pass
    return {}


# ------------------------------------------------------------ measurements

def dos_grid(emin: float, emax: float, n_moments: int):
    """ComputeDos's grid for the dE that n_moments resolves (observables.hpp:
    346-375): dE = 7.396 * half_width / N, nt = ceil(span / dE)."""
    hw = (emax - emin) / 2
    de = math.sqrt(8 * math.log(2)) * math.pi * hw / n_moments
    nt = max(1, math.ceil((emax - emin) / de))
    i = np.arange(nt)
    return np.concatenate([(i - nt) / nt, i / nt]), nt


def run_moments(wl, cheby, psi, dist):
    from rsatb_b200.calc import kpm_dos_moments
    from rsatb_b200.shard import combine_average
    mu = kpm_dos_moments(cheby, psi, wl.n_moments)
    if dist.world > 1:
        mu = combine_average(mu, wl.R, dist.sum_array, wl.R * dist.world)
    return mu


def time_recurrence(wl, precision, steps, warmup, dist):
    """(ms per step, max over ranks; moments of the last step; kernel
    launches per step)."""
    import torch
    cheby = wl.cheby64 if precision == "f64" else wl.cheby32
    psi = wl.psi(wl.vec_dtype(precision))
    for _ in range(warmup):
        mu = run_moments(wl, cheby, psi, dist)
    torch.cuda.synchronize()
    dist.barrier()
    ctx = cheby.H.ctx
    l0 = ctx.launch_count()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(steps):
        mu = run_moments(wl, cheby, psi, dist)
    e.record()
    torch.cuda.synchronize()
    dist.barrier()
    launches = (ctx.launch_count() - l0) / steps
    ms = dist.max(s.elapsed_time(e) / steps)
    return ms, mu, launches


def time_e2e(wl, precision, steps, dist):
    """Same recurrence with the sample panel copied from pinned host memory
    every step and the moments returned to the host by the C-ABI call."""
    import torch
    cheby = wl.cheby64 if precision == "f64" else wl.cheby32
    host = wl.psi(wl.vec_dtype(precision)).cpu().pin_memory()
    dev = torch.empty_like(host, device="cuda")
    torch.cuda.synchronize()
    dist.barrier()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(steps):
        dev.copy_(host, non_blocking=True)
        run_moments(wl, cheby, dev, dist)
    e.record()
    torch.cuda.synchronize()
    dist.barrier()
    ms = dist.max(s.elapsed_time(e) / steps)
    n_dot_slots = 1 + wl.n_moments // 2
    W = wl.R * (2 if wl.complex_vectors else 1)
    return ms, host.numel() * host.element_size(), n_dot_slots * 2 * W * 8


def time_spmm(A, n_rows, R, dtype, reps=20):
    """Average duration (ms) of one mult_dense launch, CUDA events."""
    import torch
    X = torch.randn(A.shape[1], R, dtype=dtype, device="cuda")
    Y = torch.empty(n_rows, R, dtype=dtype, device="cuda")
    for _ in range(3):
        A.mult_dense(X, Y)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        A.mult_dense(X, Y)
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def roofline(wl, hbm_peak, peak_note, fma_peaks):
    """Dominant kernel: the fused block SpMM of the sandwich at the run's
    panel width (each of the 3 SpMMs per application is this kernel)."""
    import torch
    from rsatb_b200.workloads import spmm_bytes, spmm_flops
    # The sandwich's SpMMs run on Z, Z^H and H (same pattern); the
    # orthogonal form on H alone.
    Z32 = wl.cheby32.M.Z if wl.cheby32.M is not None else wl.cheby32.H
    dt = wl.vec_dtype("f32")
    item = torch.empty(0, dtype=dt).element_size()
    ms = time_spmm(Z32, wl.n_rows, wl.R, dt)
    nbytes = spmm_bytes(Z32, wl.R, item)
    flops = spmm_flops(Z32, wl.R, wl.complex_vectors)
    gbs = nbytes / (ms * 1e-3) / 1e9
    tfs = flops / (ms * 1e-3) / 1e12
    # DRAM bytes (read + write) of one launch of this kernel at this shape
    # (diamond 16^3, 8x8 blocks, R = 128, FP32), from an ncu capture of that
    # launch; a profiler counter, so not measured inside this run.
    traffic = None
    if wl.n_rows == 262144 and wl.R == 128 and wl.H.block_size == 8 and not wl.complex_vectors:
        traffic = 403398400 + 118504192
    peak32 = max(fma_peaks["f32"], fma_peaks["f32x2"])
    out = {"bound": "hbm", "achieved": round(gbs, 1), "peak": hbm_peak, "unit": "GB/s",
           "frac": round(gbs / hbm_peak, 4), "traffic": traffic,
           "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch "
                             "at this shape (a separate profiled run, not this one)"
                             if traffic else None,
           "kernel": "fused BSR Chebyshev step, Y = A X, FP32, R=%d, %dx%d blocks" % (
               wl.R, wl.H.block_size, wl.H.block_size),
           "algorithmic_bytes_per_launch": nbytes, "ms_per_launch": round(ms, 4),
           "peak_source": peak_note,
           "compute": {"bound": "fp32_fma", "achieved": round(tfs, 2),
                       "peak": round(peak32 / 1e12, 2), "unit": "TFLOP/s",
                       "frac": round(tfs * 1e12 / peak32, 4),
                       "flops_per_launch": flops,
                       "peak_scalar_fma": round(fma_peaks["f32"] / 1e12, 2),
                       "peak_packed_f32x2": round(fma_peaks["f32x2"] / 1e12, 2),
                       "peak_source": "rsatb_measure_fma_peak, this run: the larger of the "
                                      "scalar and the packed (f32x2) FMA-chain rates"}}
    # The same SpMM in FP64, and the memory-bound narrow panels.
    Z64 = wl.cheby64.M.Z if wl.cheby64.M is not None else wl.cheby64.H
    dt64 = wl.vec_dtype("f64")
    ms64 = time_spmm(Z64, wl.n_rows, wl.R, dt64)
    out["fp64_same_kernel"] = {
        "ms_per_launch": round(ms64, 4),
        "gbs": round(spmm_bytes(Z64, wl.R, 2 * item) / (ms64 * 1e-3) / 1e9, 1),
        "tflops": round(spmm_flops(Z64, wl.R, wl.complex_vectors) / (ms64 * 1e-3) / 1e12, 2),
        "fma_frac": round(spmm_flops(Z64, wl.R, wl.complex_vectors) / (ms64 * 1e-3)
                          / fma_peaks["f64"], 4)}
    sweep = {}
    for R in (8, 16):
        for prec, A in (("f32", Z32), ("f64", Z64)):
            d = torch.float32 if prec == "f32" else torch.float64
            m = time_spmm(A, wl.n_rows, R, d)
            b = spmm_bytes(A, R, torch.empty(0, dtype=d).element_size())
            g = b / (m * 1e-3) / 1e9
            sweep[f"{prec}_R{R}"] = {"gbs": round(g, 1), "frac": round(g / hbm_peak, 4),
                                     "ms": round(m, 4)}
    out["hbm_sweep_narrow_panels"] = sweep
    return out


def cpu_baseline(wl, n_moments: int):
    """The oracle's FP64 recurrence (oracle/kpm_oracle.c) on the host cores,
    on the same operator and samples, over a bounded number of moments."""
    import oracle
    H = oracle.Bsr(wl.H.n_block_rows, wl.H.n_block_rows, wl.H.block_size, wl.H.row_ptr,
                   wl.H.col_ind, wl.H.values)
    if wl.Z is not None:
        Z = oracle.Bsr(wl.Z.n_block_rows, wl.Z.n_block_rows, wl.Z.block_size, wl.Z.row_ptr,
                       wl.Z.col_ind, wl.Z.values)
        op = oracle.make_op(H, (wl.emax + wl.emin) / 2, (wl.emax - wl.emin) / 2, Z,
                            oracle.bsr_adjoint(Z))
    else:
        op = oracle.make_op(H, (wl.emax + wl.emin) / 2, (wl.emax - wl.emin) / 2)
    n_atoms = wl.n_rows // wl.orbitals
    psi = oracle.set_random(20240917, 0 if wl.complex_vectors else 1, True,
                            np.arange(n_atoms), wl.orbitals, wl.n_rows, wl.R,
                            wl.complex_vectors, first_column=wl.first_column)
    t0 = time.perf_counter()
    mu = oracle.kpm_moments(op, psi, n_moments)
    dt = time.perf_counter() - t0
    return {"value": n_moments * wl.R / dt, "unit": UNIT, "cores": oracle.num_threads(),
            "kind": "port", "seconds": round(dt, 3),
            "sample": f"{n_moments} moments ({(n_moments + 1) // 2} operator applications) of "
                      f"the same workload, all {wl.R} vectors, FP64, OpenMP"}, mu


def ed_moments(dense, psi, center, half_width, n_moments):
    """KPM moments of a dense Hermitian operator on the sample columns psi by
    exact diagonalisation (numpy eigh, FP64): mu_n = (1/R) sum_q sum_k
    |(U^H psi_q)_k|^2 T_n(x_k), the rounding-free limit of the recurrence."""
    x, U = np.linalg.eigh((dense - center * np.eye(dense.shape[0])) / half_width)
    w = (np.abs(U.conj().T @ psi) ** 2).mean(axis=1)
    th = np.arccos(np.clip(x, -1.0, 1.0))
    return np.cos(np.arange(n_moments)[:, None] * th[None, :]) @ w


def dos_errors_vs_ed() -> dict:
    """Peak-normalised DOS error of the FP64 and the mixed recurrence against
    FP64 exact diagonalisation, on the same seeded samples: the graphene DOS
    configuration at full size (60 x 60, 7,200 orbitals, R = 8, 512
    moments) and a diamond LCAO sandwich (L = 3, 1,728 orbitals, R = 16, 256
    moments, Z the graph-local factor).  The headline's 262,144 orbitals are
    beyond a dense diagonalisation."""
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.calc import (Chebyshev, ISQRTMPreconditioner, evaluate_kpm_density,
                                 kpm_dos_moments)
    from rsatb_b200.isqrt import graph_inverse_sqrt
    from rsatb_b200.vbcsr import BlockSpMat, set_random
    x = np.linspace(-0.999, 0.999, 2001)

    def errs(cheby, psi, dense, n):
        t0 = time.perf_counter()
        ref = ed_moments(dense, psi.cpu().numpy(), cheby.center, cheby.half_width, n)
        rho_ref = evaluate_kpm_density(ref.astype(np.complex128), x, 1e-3)
        lo = torch.complex64 if psi.is_complex() else torch.float32
        out = {"ed_seconds": round(time.perf_counter() - t0, 2)}
        for name, c, p in (("fp64", cheby, psi), ("mixed", cheby.astype("f32"), psi.to(lo))):
            rho = evaluate_kpm_density(kpm_dos_moments(c, p, n), x, 1e-3)
            out[name] = float(np.abs(rho - rho_ref).max() / np.abs(rho_ref).max())
        return out

    H, _, _ = lattice.graphene(60, 60)
    g = Chebyshev(BlockSpMat(H.row_ptr, H.col_ind, H.values, 1), -8.6, 8.6)
    psi = torch.empty(H.n_rows, 8, dtype=torch.complex128, device="cuda")
    set_random(psi, 20240917)
    out = {"graphene_60x60_R8_512": errs(g, psi, H.to_dense(), 512)}
    Hd, S = lattice.diamond_lcao(L=3, seed=7)
    Z = graph_inverse_sqrt(S)
    torch.cuda.synchronize()
    Zd = Z.to_dense()
    op = Zd.T @ Hd.to_dense() @ Zd
    w = np.linalg.eigvalsh(op)
    d = Chebyshev(BlockSpMat(Hd.row_ptr, Hd.col_ind, Hd.values, 8), w[0] - 0.5, w[-1] + 0.5,
                  preconditioner=ISQRTMPreconditioner(BlockSpMat(Z.row_ptr, Z.col_ind, Z.values,
                                                                 8)))
    psi = torch.empty(Hd.n_rows, 16, dtype=torch.float64, device="cuda")
    set_random(psi, 20240917, orbitals_per_atom=8)
    out["diamond_L3_sandwich_R16_256"] = errs(d, psi, op, 256)
    return out


def fma_peaks() -> dict:
    import ctypes as C
    from rsatb_b200 import _capi
    from rsatb_b200.vbcsr import context
    ctx = context()
    out = {}
    for name, dp in (("f64", 1), ("f32", 0), ("f32x2", 2), ("f64_dmma", 3), ("tf32_mma", 4)):
        v = C.c_double()
        _capi.check(_capi.lib().rsatb_measure_fma_peak(ctx.handle, dp, C.byref(v)))
        out[name] = v.value
    return out


def build_workload(args, rank):
    from rsatb_b200 import workloads
    if args.workload == "graphene":
        return workloads.graphene_dos(30 if args.small else 60, 30 if args.small else 60,
                                      rank=rank)
    if args.small:
        return workloads.diamond_sandwich(L=6, R=32, n_moments=256, rank=rank)
    return workloads.diamond_sandwich(rank=rank)


def config_of(wl) -> dict:
    """The workload as both arms name it (the spectral window, which each
    arm estimates for itself, is reported beside the config)."""
    return {"workload": wl.name + (": diamond LCAO %d^3 conventional cells, %d atoms x 8 "
                                   "orbitals, 8x8 BSR to the 3rd shell (29 blocks/row), "
                                   "operator Z^H H Z with the graph-local S^-1/2"
                                   % (round((wl.n_rows // 64) ** (1 / 3)), wl.n_rows // 8)
                                   if wl.name == "diamond_sandwich" else ": pz graphene"),
            "n_rows": wl.n_rows, "vectors_per_gpu": wl.R, "n_moments": wl.n_moments,
            "block_size": wl.H.block_size, "nnz_blocks": int(wl.H.nnz_blocks),
            "sample_vectors": "complex random phase" if wl.complex_vectors else "Rademacher",
            "l2": "inputs larger than L2 (every panel >= 134 MB > 126 MB L2)"
            if wl.n_rows * wl.R * 4 > 126e6 else "working set may be L2-resident"}


class HostWorkload:
    """The bench workload built on the host only (numpy and the oracle), for
    the reference arm: the same seeded H (and S), the graph-local S^-1/2 by
    the reference's eigen route, the spectral window by the same Lanczos
    from the same start vector, the same sample vectors.  Nothing here loads
    the CUDA library."""

    def __init__(self, args):
        import oracle
        from rsatb_b200 import lattice
        t0 = time.perf_counter()
        self.setup_seconds = {}
        self.first_column = 0
        if args.workload == "graphene":
            n = 30 if args.small else 60
            self.name, self.R, self.n_moments, self.orbitals = "graphene_dos", 8, 512, 1
            self.complex_vectors = True
            self.H, _, _ = lattice.graphene(n, n)
            self.Z = None
        else:
            L, self.R, self.n_moments = (6, 32, 256) if args.small else (16, 128, 1024)
            self.name, self.orbitals, self.complex_vectors = "diamond_sandwich", 8, False
            self.H, S = lattice.diamond_lcao(L=L, seed=7)
            self.setup_seconds["generate"] = time.perf_counter() - t0
            t1 = time.perf_counter()
            zv = oracle.graph_inverse_sqrt_eigen(S.row_ptr, S.col_ind, S.values, S.block_size)
            self.Z = lattice.BsrArrays(S.row_ptr, S.col_ind, zv, S.block_size)
            self.setup_seconds["graph_inverse_sqrt_eigen"] = time.perf_counter() - t1
        t1 = time.perf_counter()
        H = oracle.Bsr(self.H.n_block_rows, self.H.n_block_rows, self.H.block_size,
                       self.H.row_ptr, self.H.col_ind, self.H.values)
        Z = ZH = None
        if self.Z is not None:
            Z = oracle.Bsr(self.Z.n_block_rows, self.Z.n_block_rows, self.Z.block_size,
                           self.Z.row_ptr, self.Z.col_ind, self.Z.values)
            ZH = oracle.bsr_adjoint(Z)
        unit = oracle.make_op(H, 0.0, 1.0, Z, ZH)
        self.emin, self.emax = oracle.lanczos_bounds(lambda X: oracle.apply_op(unit, X),
                                                     self.H.n_rows)
        self.setup_seconds["lanczos_bounds"] = time.perf_counter() - t1

    @property
    def n_rows(self) -> int:
        return self.H.n_rows


def reference_arm(args):
    """The reference's CPU path on the host cores, rank 0 only: the oracle's
    FP64 restatement of the recurrence (the reference itself cannot be built
    here), timed over the same number of moments as the cpu_baseline leg, on
    a workload built on the host without the CUDA library."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    if args.workload not in ("diamond", "graphene"):
        print(json.dumps({"impl": "reference",
                          "unavailable": "the reference arm covers the KPM DOS workloads "
                                         "(diamond, graphene); the --workload %s line carries "
                                         "its own cpu_baseline" % args.workload}), flush=True)
        return
    wl = HostWorkload(args)
    n_mom = args.cpu_moments
    samples = []
    for k in range(args.warmup + args.steps):
        base, _ = cpu_baseline(wl, n_mom)
        if k >= args.warmup:
            samples.append(base)
    secs = [s["seconds"] for s in samples]
    value = n_mom * wl.R / (sum(secs) / len(secs))
    base = dict(samples[-1])
    base["value"] = value
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(secs) / len(secs), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(wl), "cpu_baseline": base,
            "bounds_ev": [round(wl.emin, 4), round(wl.emax, 4)],
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "cuda_library_loaded": "rsatb_b200._capi" in sys.modules,
            "setup_seconds": {k: round(v, 2) for k, v in wl.setup_seconds.items()},
            "note": "RSATB cannot be built here (vbcsr, PRIMME, MPI, FFTW, HDF5 absent); the "
                    "timed CPU path is the oracle's FP64 restatement of the same recurrence, "
                    "on H, Z (eigen route) and the window built on the host"}
    print(json.dumps(line), flush=True)


def spmm_only(args):
    """Y = H X on the diamond H at R = 128 and R = 8, FP32 and FP64: the
    small case the ncu captures of the step kernel use (every operand above
    the 126 MB L2 for R = 128)."""
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.vbcsr import BlockSpMat
    from rsatb_b200.workloads import spmm_bytes, spmm_flops
    H, _ = lattice.diamond_lcao(L=args.spmm_L, seed=7)
    A64 = BlockSpMat(H.row_ptr, H.col_ind, H.values, 8)
    A32 = A64.astype("f32")
    out = {"n_rows": H.n_rows, "nnz_blocks": int(H.nnz_blocks)}
    widths = [int(r) for r in args.spmm_widths.split(",") if r]
    if args.spmm_kernels:
        # A/B of the FP32 step kernels: time and max error against the FP64
        # SpMM of the same (FP32-representable) panel.
        for R in widths:
            torch.manual_seed(R)
            X = torch.randn(H.n_rows, R, dtype=torch.float32, device="cuda")
            Y64 = torch.empty(H.n_rows, R, dtype=torch.float64, device="cuda")
            A64.mult_dense(X.double(), Y64)
            ref = Y64.cpu()
            for k in args.spmm_kernels.split(","):
                kind, _, shape = k.partition(":")
                os.environ["RSATB_STEP_KERNEL"] = kind
                if shape:
                    os.environ["RSATB_TF32_SHAPE"] = shape
                ms = time_spmm(A32, H.n_rows, R, torch.float32, reps=max(args.spmm_reps, 20))
                Y = torch.empty(H.n_rows, R, dtype=torch.float32, device="cuda")
                A32.mult_dense(X, Y)
                err = float((Y.double().cpu() - ref).abs().max() / ref.abs().max())
                out[f"f32_R{R}_{k}"] = {"ms": round(ms, 4), "rel_err_vs_fp64": err}
                os.environ.pop("RSATB_STEP_KERNEL", None)
                os.environ.pop("RSATB_TF32_SHAPE", None)
        print(json.dumps(out), flush=True)
        return
    for R in widths:
        for name, A, dt in (("f32", A32, torch.float32), ("f64", A64, torch.float64)):
            ms = time_spmm(A, H.n_rows, R, dt, reps=args.spmm_reps)
            b = spmm_bytes(A, R, torch.empty(0, dtype=dt).element_size())
            out[f"{name}_R{R}"] = {"ms": round(ms, 4), "gbs": round(b / ms / 1e6, 1),
                                   "tflops": round(spmm_flops(A, R, False) / ms / 1e9, 2)}
    print(json.dumps(out), flush=True)


def forms_only(args):
    """Cost of one operator application in the Sandwich form Z^H H Z and in
    the Solve form S^-1 H (CG with S, plain and preconditioned by the
    graph-local Z), the comparison the reference quotes for diamond
    (rsatb/model/setup.hpp:44-47: the sandwich 5.9x faster per matvec).
    Diamond LCAO L^3 cells, 8x8 blocks, R = 16 real vectors, FP64; each
    application starts its CG from zero."""
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.bounds import estimate_spectral_bounds
    from rsatb_b200.calc import Chebyshev, ISQRTMPreconditioner, cg_solve
    from rsatb_b200.isqrt import graph_inverse_sqrt
    from rsatb_b200.vbcsr import BlockSpMat, set_random
    H, S = lattice.diamond_lcao(L=args.forms_L, seed=7)
    Z = graph_inverse_sqrt(S, method="ns")
    dev = lambda A: BlockSpMat(A.row_ptr, A.col_ind, A.values, A.block_size)
    Hd, Sd = dev(H), dev(S)
    pre = ISQRTMPreconditioner(dev(Z))
    emin, emax = estimate_spectral_bounds(Chebyshev(Hd, -1.0, 1.0, preconditioner=pre))
    forms = {"sandwich": Chebyshev(Hd, emin, emax, preconditioner=pre),
             "solve_cg": Chebyshev(Hd, emin, emax, overlap=Sd),
             "solve_pcg_z": Chebyshev(Hd, emin, emax, overlap=Sd, preconditioner=pre)}
    R = 16
    X = torch.empty(H.n_rows, R, dtype=torch.float64, device="cuda")
    set_random(X, 3)
    Y = torch.empty_like(X)
    out = {"n_rows": H.n_rows, "R": R, "nnz_blocks": int(H.nnz_blocks)}
    for name, c in forms.items():
        for _ in range(2):
            Y.zero_()
            c.apply_op(X, Y)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(args.spmm_reps):
            Y.zero_()
            c.apply_op(X, Y)
        e.record()
        torch.cuda.synchronize()
        out[f"{name}_ms"] = round(s.elapsed_time(e) / args.spmm_reps, 4)
    B = torch.empty_like(X)
    Hd.mult_dense(X, B)
    for name, p in (("cg", None), ("pcg_z", pre)):
        Xs = torch.zeros_like(X)
        it, res = cg_solve(Sd, B, Xs, tol=1e-8, max_iter=1000, preconditioner=p)
        out[f"{name}_iterations"] = it
    out["solve_cg_over_sandwich"] = round(out["solve_cg_ms"] / out["sandwich_ms"], 2)
    out["solve_pcg_z_over_sandwich"] = round(out["solve_pcg_z_ms"] / out["sandwich_ms"], 2)
    print(json.dumps(out), flush=True)


def bench_isqrt(args, dist):
    """Batched graph-local S^-1/2: args.isqrt_n SPD problems per GPU, sizes
    uniform in [40, 400], condition numbers log-uniform in [1e2, 1e5]; each
    problem returns 16 columns of its inverse square root from column n/3
    (an interior block row, as the graph-local factor takes).  One step =
    one rsatb_isqrt_columns_batched call over the whole batch."""
    import torch
    import oracle
    from rsatb_b200 import workloads
    from rsatb_b200.isqrt import inverse_sqrt_columns_batched
    t0 = time.perf_counter()
    batch = workloads.batched_spd(args.isqrt_n, family=args.isqrt_family, seed=7 + dist.rank)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    n = batch.n
    cs = (n // 3).astype(np.int32)
    ks = np.minimum(16, n - cs).astype(np.int32)
    out_off = np.concatenate([[0], np.cumsum(n.astype(np.int64) * ks)[:-1]]).astype(np.int64)
    out = torch.zeros(int((n.astype(np.int64) * ks).sum()), dtype=torch.float64, device="cuda")
    ws = int(args.isqrt_ws_gb * (1 << 30))

    # Tensor-core tiles from the autotuner (seeded samples of every padded
    # size in the batch), picked before and outside the timed region.
    tiles, tune_s = None, 0.0
    if args.isqrt_precision != "fp64" and not args.isqrt_no_autotune:
        from rsatb_b200.isqrt import autotune_tiles
        t1 = time.perf_counter()
        tiles = autotune_tiles(np.unique(n), precision=args.isqrt_precision,
                               problems_per_size=16)
        tune_s = time.perf_counter() - t1

    def run(prec):
        return inverse_sqrt_columns_batched(batch.flat, n, batch.offset, cs, ks, out_off,
                                            precision=prec, out=out, workspace_bytes=ws,
                                            tiles=tiles if prec != "fp64" else None)

    def timed(prec, steps, warmup):
        for _ in range(warmup):
            run(prec)
        torch.cuda.synchronize()
        dist.barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        for _ in range(steps):
            _, status, stats = run(prec)
        ev[1].record()
        torch.cuda.synchronize()
        dist.barrier()
        return dist.max(ev[0].elapsed_time(ev[1]) / steps), status, stats

    peaks = measured_peaks()
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms, status, stats = timed(args.isqrt_precision, args.steps, args.warmup)
    clocks = clk.summary()
    host = out.cpu().numpy()
    rng = np.random.default_rng(1)
    sample = rng.choice(n.size, size=min(48, n.size), replace=False)
    err = 0.0
    for p in sample:
        want = oracle.isqrt_columns_eigen(batch.matrix(p), int(cs[p]), int(ks[p]))
        got = host[out_off[p]:out_off[p] + n[p] * ks[p]].reshape(ks[p], n[p]).T
        err = max(err, float(np.linalg.norm(got - want) / np.linalg.norm(want)))
    ms64 = None
    if args.isqrt_precision != "fp64":
        ms64, _, stats64 = timed("fp64", 1, 0)
    fma = fma_peaks()
    f64_peak = max(fma["f64"], fma["f64_dmma"])
    tf32_peak = 0.5 * float(peaks.get("bf16_tflops", 1590.0))
    low_tfs = stats["low_flops"] / max(stats["low_ms"], 1e-9) / 1e9
    f64_tfs = stats["fp64_flops"] / max(stats["fp64_ms"], 1e-9) / 1e9
    units = n.size * dist.world
    if dist.rank == 0:
        line = {
            "metric": "batched graph-local S^-1/2 throughput", "value": round(units / (ms * 1e-3), 1),
            "unit": "matrices/s", "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"tf32x3": "split TF32 (FP32 accumulate) + FP64 refinement",
                      "tf32": "TF32 (FP32 accumulate) + FP64 refinement",
                      "fp64": "f64"}[args.isqrt_precision],
            "data": f"synthetic (seeded Q diag(l) Q^T, {args.isqrt_family} spectra)",
            "config": {"workload": "batched_isqrt: SPD n~U[40,400], kappa log-uniform "
                                   "[1e2,1e5], 16 columns from n/3 per problem",
                       "spectrum_family": args.isqrt_family,
                       "problems_per_gpu": int(n.size), "sum_n_cubed": float((n.astype(
                           np.float64) ** 3).sum()), "workspace_gb_per_chunk": args.isqrt_ws_gb},
            "status_failures": int((status != 0).sum()),
            "max_rel_err_vs_eigh_sample": err, "sample_size": int(sample.size),
            "stats": {k: (float(f"{v:.4g}") if isinstance(v, float) else v)
                      for k, v in stats.items()},
            "roofline": {"bound": "tensor", "achieved": round(low_tfs, 1),
                         "peak": round(tf32_peak, 1), "unit": "TFLOP/s",
                         "frac": round(low_tfs / tf32_peak, 4), "traffic": None,
                         "kernel": "tc_gemm_ws_kernel (tcgen05 kind::tf32, executed tile "
                                   "FLOPs over the whole tensor-core phase, FP64 updates "
                                   "included in its time)",
                         "peak_source": "MEASURED_PEAKS.json bf16_tflops / 2 (dense TF32 rate)",
                         "fp64_phase": {"kernel": "gemm_f64_kernel (mma.sync m8n8k4 f64, "
                                                  "cp.async double-buffered)",
                                        "achieved": round(f64_tfs, 2),
                                        "peak": round(f64_peak / 1e12, 2),
                                        "frac": round(f64_tfs * 1e12 / f64_peak, 4),
                                        "peak_source": "rsatb_measure_fma_peak, this run: the "
                                                       "larger of the FP64 FMA-chain and the "
                                                       "m8n8k4 tensor-chain rates",
                                        "peak_fp64_fma": round(fma["f64"] / 1e12, 2),
                                        "peak_fp64_tensor": round(fma["f64_dmma"] / 1e12, 2)}},
            "fp64_only_ms_per_step": round(ms64, 2) if ms64 else None,
            "speedup_vs_fp64_only": round(ms64 / ms, 3) if ms64 else None,
            "clocks": clocks, "generate_seconds": round(gen_s, 1),
            "autotuned_tiles": None if tiles is None else {
                "tc_kernel": "warp-specialised" if tiles.tc_kernel == 1 else "single-role",
                "n_tile_per_n_pad": tiles.nt, "tune_seconds": round(tune_s, 1)},
        }
        print(json.dumps(line), flush=True)


def bench_transport(args, dist):
    """Kubo-Greenwood sigma(E) by FFT-Chebyshev on twisted bilayer graphene
    (commensurate moire cell m, tiled tiles x tiles; pz, NN intralayer
    t = -2.7 eV, interlayer 0.48 exp(-(d - 3.35)/0.45) within 6 A), commutator
    velocities at Gamma, random-phase samples sharded over the GPUs.  One step
    = one dc_spectrum_fftcheb call over this GPU's samples: FP32 vectors with
    the fused row stage's FP32 transform with FP64 products and sums; the FP64
    path is timed beside it."""
    import torch
    import oracle
    from rsatb_b200 import lattice
    from rsatb_b200.bounds import estimate_spectral_bounds
    from rsatb_b200.calc import Chebyshev
    from rsatb_b200.transport import dc_spectrum_fftcheb
    from rsatb_b200.vbcsr import BlockSpMat, set_random
    t0 = time.perf_counter()
    H, pos, cell, disp = lattice.twisted_bilayer_graphene(m=args.tbg_m,
                                                         tiles=(args.tbg_tiles, args.tbg_tiles))
    V = lattice.commutator_velocity(H, disp)
    gen_s = time.perf_counter() - t0
    c0 = Chebyshev(BlockSpMat(H.row_ptr, H.col_ind, H.values, 1), -1.0, 1.0)
    emin, emax = estimate_spectral_bounds(c0)
    c64 = Chebyshev(c0.H, emin, emax)
    c32 = c64.astype("f32")
    V64 = [BlockSpMat(v.row_ptr, v.col_ind, v.values, 1, imaginary=True) for v in V]
    V32 = [v.astype("f32") for v in V64]
    R = max(1, args.transport_samples // dist.world)
    M = args.transport_moments
    psi64 = torch.empty(H.n_rows, R, dtype=torch.complex128, device="cuda")
    set_random(psi64, 20240917, normalize=True, orbitals_per_atom=1, kind=0,
               first_column=dist.rank * R)
    psi32 = psi64.to(torch.complex64)

    def timed(c, Vs, psi, steps, warmup):
        for _ in range(warmup):
            dc_spectrum_fftcheb(c, *Vs, psi, M)
        torch.cuda.synchronize()
        dist.barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        for _ in range(steps):
            out = dc_spectrum_fftcheb(c, *Vs, psi, M, return_stats=True)
        ev[1].record()
        torch.cuda.synchronize()
        dist.barrier()
        return dist.max(ev[0].elapsed_time(ev[1]) / steps), out

    with ClockSampler(torch.cuda.current_device()) as clk:
        ms32, (sig32, energy, st32) = timed(c32, V32, psi32, args.steps, args.warmup)
    clocks = clk.summary()
    ms64, (sig64, _, st64) = timed(c64, V64, psi64, 1, 0)
    sig32 = dist.sum_array(sig32 * R) / (R * dist.world)
    sig64 = dist.sum_array(sig64 * R) / (R * dist.world)
    diag = [0, 3, 5]
    err = float(np.abs(sig32[:, diag] - sig64[:, diag]).max() / np.abs(sig64[:, diag]).max())
    base = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        # Bounded CPU sample: one moire cell (no tiling), 2 samples, 128 moments.
        Hs, _, _, ds = lattice.twisted_bilayer_graphene(m=args.tbg_m, tiles=(1, 1))
        Vs = [oracle.Bsr(h.n_block_rows, h.n_block_rows, 1, h.row_ptr, h.col_ind, h.values,
                         imag=True) for h in lattice.commutator_velocity(Hs, ds)]
        op = oracle.make_op(oracle.Bsr(Hs.n_block_rows, Hs.n_block_rows, 1, Hs.row_ptr,
                                       Hs.col_ind, Hs.values), (emax + emin) / 2,
                            (emax - emin) / 2)
        ps = np.exp(2j * np.pi * np.random.default_rng(0).random((Hs.n_rows, 2))) / math.sqrt(
            Hs.n_rows)
        tc = time.perf_counter()
        oracle.fftcheb(op, Vs, ps, 128)
        dt = time.perf_counter() - tc
        base = {"value": 2 * 128 * Hs.n_rows / dt, "unit": "sample-moment-rows/s",
                "cores": oracle.num_threads(), "kind": "port", "seconds": round(dt, 3),
                "sample": f"one moire cell ({Hs.n_rows} atoms), 2 samples, 128 moments, FP64"}
    units = R * dist.world * M
    if dist.rank == 0:
        line = {
            "metric": "Kubo-Greenwood sigma(E) by FFT-Chebyshev", "value": round(units / (
                ms32 * 1e-3), 1), "unit": "sample-moments/s", "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms32, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 vectors and transform, FP64 contraction sums",
            "data": "synthetic (seeded TBG generator, random phases)",
            "config": {"workload": f"transport_tbg: m={args.tbg_m} moire cell tiled "
                                   f"{args.tbg_tiles}x{args.tbg_tiles}",
                       "n_rows": H.n_rows, "nnz": int(H.nnz_blocks), "n_moments": M,
                       "samples_per_gpu": R, "bounds_ev": [round(emin, 4), round(emax, 4)]},
            "stats_f32": st32, "fp64_path": {"ms_per_step": round(ms64, 2), "stats": st64,
                                             "mixed_over_fp64": round(ms64 / ms32, 3)},
            "sigma_err_f32_vs_f64": err, "cpu_baseline": base,
            "throughput_rows_per_s": round(units * H.n_rows / (ms32 * 1e-3), 1),
            "clocks": clocks, "generate_seconds": round(gen_s, 1)}
        print(json.dumps(line), flush=True)


def bench_adjoint(args, dist):
    """Adjoint KPM on silicon sp3s* (L^3 conventional cells, 5x5 blocks to the
    2nd shell, N(0, 0.1) eV around fixed SK-like means): loss = L2 between the
    Jackson DOS (256 moments, 32 Rademacher vectors per GPU, 1001 energies)
    and the DOS of a second seeded silicon sample; one step = loss forward +
    gradient with respect to all block values (autograd backward through the
    checkpointed adjoint recurrence)."""
    import torch
    import oracle
    from rsatb_b200 import lattice
    from rsatb_b200.adjoint import KpmDosLoss, dos_basis, kpm_moments_vjp
    from rsatb_b200.bounds import estimate_spectral_bounds
    from rsatb_b200.calc import Chebyshev, kpm_dos_moments_plain
    from rsatb_b200.vbcsr import BlockSpMat, set_random
    M, R = 256, 32
    H = lattice.silicon_sp3s(L=args.si_L, seed=11)
    Ht = lattice.silicon_sp3s(L=args.si_L, seed=12)
    Hd = BlockSpMat(H.row_ptr, H.col_ind, H.values, 5)
    Htd = BlockSpMat(Ht.row_ptr, Ht.col_ind, Ht.values, 5)
    e1 = estimate_spectral_bounds(Chebyshev(Hd, -1, 1))
    e2 = estimate_spectral_bounds(Chebyshev(Htd, -1, 1))
    emin, emax = min(e1[0], e2[0]), max(e1[1], e2[1])
    psi = torch.empty(H.n_rows, R, dtype=torch.float64, device="cuda")
    set_random(psi, 20240917, normalize=True, orbitals_per_atom=5, kind=1,
               first_column=dist.rank * R)
    x = np.linspace(-0.98, 0.98, 1001)
    D = dos_basis(M, x)
    target = D @ kpm_dos_moments_plain(Chebyshev(Htd, emin, emax), psi, M).real
    v0 = torch.as_tensor(H.values).cuda()

    def step():
        v = v0.clone().requires_grad_(True)
        loss = KpmDosLoss.apply(v, Hd, psi, emin, emax, M, x, target)
        loss.backward()
        return float(loss), v.grad

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    dist.barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    with ClockSampler(torch.cuda.current_device()) as clk:
        ev[0].record()
        for _ in range(args.steps):
            loss, g = step()
        ev[1].record()
        torch.cuda.synchronize()
    clocks = clk.summary()
    ms = dist.max(ev[0].elapsed_time(ev[1]) / args.steps)
    dist.barrier()
    # FD checks (h = 1e-6): 6 sampled values and one random direction.
    h = 1e-6
    rng = np.random.default_rng(3)

    def L(vals):
        return float(KpmDosLoss.apply(vals, Hd, psi, emin, emax, M, x, target))

    flat = v0.reshape(-1)
    fd_err = 0.0
    gf = g.reshape(-1).cpu().numpy()
    gscale = float(np.abs(gf).max())
    for e in rng.choice(flat.numel(), size=6, replace=False):
        p, m_ = flat.clone(), flat.clone()
        p[e] += h
        m_[e] -= h
        fd = (L(p.view_as(v0)) - L(m_.view_as(v0))) / (2 * h)
        fd_err = max(fd_err, abs(fd - gf[e]) / gscale)
    Dv = torch.as_tensor(rng.standard_normal(tuple(v0.shape))).cuda()
    fd = (L(v0 + h * Dv) - L(v0 - h * Dv)) / (2 * h)
    an = float((g * Dv).sum())
    dir_err = abs(fd - an) / max(abs(an), 1e-300)
    # FP32 vectors against the FP64 gradient (same dmu).
    Hd.set_values(v0)
    c64 = Chebyshev(Hd, emin, emax)
    mu = kpm_dos_moments_plain(c64, psi, M).real
    dmu = 2.0 * ((D @ mu - target) @ D)
    g64, _, st64 = kpm_moments_vjp(c64, psi, M, dmu)
    g32, _, st32 = kpm_moments_vjp(c64.astype("f32"), psi.float(), M, dmu)
    err32 = float((g32 - g64).abs().max() / g64.abs().max())
    base = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        import scipy.sparse as sp
        Hcsr = sp.csr_matrix(H.to_dense()) if H.n_rows <= 4000 else None
        if Hcsr is None:
            rows = np.repeat(np.arange(H.n_block_rows), np.diff(H.row_ptr))
            b = 5
            rr = (rows[:, None, None] * b + np.arange(b)[None, :, None]).repeat(b, 2)
            cc = (H.col_ind[:, None, None] * b + np.arange(b)[None, None, :]).repeat(b, 1)
            Hcsr = sp.csr_matrix((H.values.reshape(-1), (rr.reshape(-1), cc.reshape(-1))),
                                 shape=(H.n_rows, H.n_rows))
        ms_cpu = 32
        tc = time.perf_counter()
        oracle.kpm_moments_vjp_sparse(Hcsr, psi.cpu().numpy(), (emax + emin) / 2,
                                      (emax - emin) / 2, ms_cpu, dmu[:ms_cpu])
        dt = time.perf_counter() - tc
        base = {"value": 1e3 * dt * M / ms_cpu, "unit": "ms per gradient (extrapolated)",
                "cores": 1, "kind": "port", "seconds": round(dt, 3),
                "sample": f"{ms_cpu} of {M} moments, same operator and samples, scipy.sparse "
                          "FP64, extrapolated linearly to 256 moments"}
    if dist.rank == 0:
        line = {
            "metric": "adjoint KPM gradient of a DOS loss", "value": round(ms, 3),
            "unit": "ms per loss+gradient", "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Si sp3s* generator, Rademacher vectors)",
            "config": {"workload": f"adjoint_si: Si {args.si_L}^3 cells sp3s*, 5x5 blocks to "
                                   "the 2nd shell", "n_rows": H.n_rows,
                       "nnz_blocks": int(H.nnz_blocks), "n_moments": M,
                       "vectors_per_gpu": R, "energies": int(x.size)},
            "loss": loss, "fd_max_err_rel_to_max_grad": fd_err, "directional_fd_rel_err": dir_err,
            "grad_f32_vs_f64_rel": err32, "vjp_stats_f64": st64, "vjp_stats_f32": st32,
            "cpu_baseline": base, "clocks": clocks}
        print(json.dumps(line), flush=True)


def spawn_ranks(args) -> int:
    """`bench.py --gpus N` started without a launcher: runs the same command
    under torch.distributed.run with N local ranks (one per GPU, rendezvous
    on 127.0.0.1), whose rank 0 prints the line; returns their exit status."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1",
           f"--master-port={port}", str(ROOT / "bench.py"), *sys.argv[1:]]
    return subprocess.run(cmd, timeout=3600).returncode


def chain_moments(n_rows: int, first_column: int, n_cols: int, n_moments: int) -> np.ndarray:
    """Host workload for the rank plumbing: plain Chebyshev moments
    mu_n = <psi|T_n(H)|psi> summed over the sample columns first_column ..
    first_column + n_cols - 1 of a periodic chain H (hopping 1/2, spectrum
    in [-1, 1]), each column seeded by its global index (numpy)."""
    cols = [np.random.default_rng(1000 + c).choice([-1.0, 1.0], n_rows) / np.sqrt(n_rows)
            for c in range(first_column, first_column + n_cols)]
    psi = np.stack(cols, axis=1)
    H = lambda x: 0.5 * (np.roll(x, 1, axis=0) + np.roll(x, -1, axis=0))
    mu = np.zeros(n_moments)
    t0, t1 = psi, H(psi)
    mu[0] = float((psi * t0).sum())
    if n_moments > 1:
        mu[1] = float((psi * t1).sum())
    for n in range(2, n_moments):
        t0, t1 = t1, 2.0 * H(t1) - t0
        mu[n] = float((psi * t1).sum())
    return mu


def bench_chain(args, dist):
    """The host-only chain workload: each rank its own R columns, one
    all-reduce of the moment sums per step, max-over-ranks time."""
    R, n_rows, n_mom = 4, 4096, 64
    for _ in range(args.warmup):
        dist.sum_array(chain_moments(n_rows, dist.rank * R, R, n_mom))
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        mu = dist.sum_array(chain_moments(n_rows, dist.rank * R, R, n_mom)) / (R * dist.world)
    secs = dist.max((time.perf_counter() - t0) / args.steps)
    if dist.rank == 0:
        print(json.dumps({"metric": "chain moments (host plumbing check)",
                          "value": n_mom * R * dist.world / secs, "unit": UNIT,
                          "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * secs, "moments": mu.tolist(),
                          "config": {"workload": "chain", "n_rows": n_rows,
                                     "vectors_per_rank": R, "n_moments": n_mom}}), flush=True)


def main():
    args = parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and args.impl == "ours":
        sys.exit(spawn_ranks(args))
    if args.spmm_only:
        spmm_only(args)
        return
    if args.forms_only:
        forms_only(args)
        return
    if args.impl == "reference":
        reference_arm(args)
        return
    dist = Dist()
    if args.workload == "chain":
        bench_chain(args, dist)
        dist.close()
        return
    if args.workload == "isqrt" and args.impl == "ours":
        bench_isqrt(args, dist)
        dist.close()
        return
    if args.workload == "adjoint" and args.impl == "ours":
        bench_adjoint(args, dist)
        dist.close()
        return
    if args.workload == "transport" and args.impl == "ours":
        bench_transport(args, dist)
        dist.close()
        return
    import torch
    from rsatb_b200.calc import evaluate_kpm_density

    wl = build_workload(args, dist.rank)
    peaks = measured_peaks()
    hbm_peak = float(peaks.get("hbm_gbs", FALLBACK_HBM_GBS))
    peak_note = ("MEASURED_PEAKS.json hbm_gbs (measured copy, burst)" if "hbm_gbs" in peaks
                 else "fallback 6650 GB/s")
    fpk = fma_peaks()

    with ClockSampler(torch.cuda.current_device()) as clk:
        ms64, mu64, _ = time_recurrence(wl, "f64", args.steps, args.warmup, dist)
        ms32, mu32, launches = time_recurrence(wl, "f32", args.steps, args.warmup, dist)
    clocks = clk.summary()
    e2e_ms, h2d, d2h = time_e2e(wl, "f32", args.steps, dist)
    roof = roofline(wl, hbm_peak, peak_note, fpk)

    x, nt = dos_grid(wl.emin, wl.emax, wl.n_moments)
    rho64 = 2 * evaluate_kpm_density(mu64, x, 0.5 / nt)
    rho32 = 2 * evaluate_kpm_density(mu32, x, 0.5 / nt)
    dos_err = float(np.abs(rho32 - rho64).max() / np.abs(rho64).max())
    ed = dos_errors_vs_ed() if dist.rank == 0 and not args.small else None

    units = wl.n_moments * wl.R * dist.world
    value = units / (ms32 * 1e-3)
    value64 = units / (ms64 * 1e-3)
    base = None
    if dist.rank == 0 and not args.no_cpu_baseline and dist.world == 1:
        base, mu_cpu = cpu_baseline(wl, args.cpu_moments)
        base["moments_vs_gpu_fp64_max_abs"] = float(np.abs(mu_cpu - mu64[:args.cpu_moments]).max())

    if dist.rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms32, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (FP64 rescale + moment dots)", "data": "synthetic (seeded generators)",
            "config": config_of(wl),
            "parallelism": f"samples sharded over {dist.world} GPU(s)",
            "bounds_ev": [round(wl.emin, 4), round(wl.emax, 4)],
            "fp64_path": {"value": round(value64, 1), "ms_per_step": round(ms64, 3),
                          "mixed_over_fp64": round(ms64 / ms32, 3)},
            "dos_err_mixed_vs_fp64": dos_err,
            "dos_err_vs_ed": ed,
            "roofline": roof,
            "cpu_baseline": base,
            "e2e": {"value": round(units / (e2e_ms * 1e-3), 1), "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": round(e2e_ms, 3)},
            "gpu_launches": int(round(launches * args.steps)),
            "launches_per_step": launches,
            "fma_peaks_tflops": {k: round(v / 1e12, 2) for k, v in fpk.items()},
            "clocks": clocks,
            "setup_seconds": {k: round(v, 2) for k, v in wl.setup_seconds.items()},
        }
        print(json.dumps(line), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
