"""Sample sharding over ranks (one process per GPU).

The KPM moments, the Kubo-Greenwood sigma(E) and the adjoint gradient are
sums over independent sample columns (rsatb/calc/dos.hpp:134-138 averages
the per-column dots; fftcheb_transport.hpp:602 all-reduces the per-rank
kappa).  Each rank takes a contiguous block of global sample columns — the
generator is keyed by the global column, so the union over ranks is the
single-process sample set — runs its block, and one all-reduce of the
sample-weighted results forms the global average.  No exchange happens
inside the recurrence: every operator fits one GPU.
"""
from __future__ import annotations

import numpy as np


def sample_block(n_total: int, world: int, rank: int) -> tuple[int, int]:
    """(first global column, number of columns) of `rank`'s block of
    n_total samples: contiguous, sizes differing by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    base, extra = divmod(n_total, world)
    count = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, count


def combine_average(local: np.ndarray, local_count: int, all_reduce_sum, total: int) -> np.ndarray:
    """Global sample average from this rank's average over local_count
    samples: all_reduce_sum(local * local_count) / total.  all_reduce_sum
    sums a real float64 array over the ranks (NCCL or gloo)."""
    a = np.asarray(local)
    if np.iscomplexobj(a):
        flat = np.concatenate([a.real.ravel(), a.imag.ravel()]) * local_count
        s = all_reduce_sum(flat)
        n = a.size
        return (s[:n] + 1j * s[n:]).reshape(a.shape) / total
    return all_reduce_sum(a.ravel() * float(local_count)).reshape(a.shape) / total


def torch_all_reduce_sum(device=None):
    """all_reduce_sum over the default torch.distributed group (float64)."""
    import torch
    import torch.distributed as dist

    def f(x: np.ndarray) -> np.ndarray:
        t = torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64))
        if device is not None:
            t = t.to(device)
        dist.all_reduce(t)
        return t.cpu().numpy()
    return f
