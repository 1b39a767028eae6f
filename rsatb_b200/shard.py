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


# ------------------------------------------------------------- k-points

def kpoint_colour(npar: int, world_rank: int, world_size: int) -> int:
    """The sub-communicator ("colour") of a rank when the k-points are
    spread over npar of them (clamped to [1, world_size])."""
    npar = max(1, min(int(npar), int(world_size)))
    return (int(world_rank) * npar) // int(world_size)


def partition_kpoints(kpoints, npar: int, world_rank: int, world_size: int):
    """PartitionKPoints (rsatb/setup/kpoint_partition.hpp:56-80): k-point i
    belongs to colour i mod npar; every rank of a colour owns the same
    k-points.  Returns [(global index, k-point), ...] in ascending index."""
    if world_size < 1:
        raise ValueError("world_size must be at least 1")
    if not 0 <= world_rank < world_size:
        raise ValueError("world_rank is outside the communicator")
    npar_c = max(1, min(int(npar), int(world_size)))
    colour = kpoint_colour(npar, world_rank, world_size)
    return [(i, k) for i, k in enumerate(kpoints) if i % npar_c == colour]


def gather_kpoint_results(values: np.ndarray, npar: int, world_rank: int, world_size: int,
                          all_reduce_sum) -> np.ndarray:
    """GatherKPointResults (rsatb/calc/observables.hpp:137-148): the global
    per-k-point array, zero where this rank owns nothing, summed over the
    first rank of every colour (the reference's master communicator) and
    shared with every rank (its broadcast within the colour).  One
    all-reduce in which only colour leaders contribute does both."""
    colour = kpoint_colour(npar, world_rank, world_size)
    leader = world_rank == 0 or kpoint_colour(npar, world_rank - 1, world_size) != colour
    v = np.asarray(values, dtype=np.float64)
    return all_reduce_sum(v.ravel() if leader else np.zeros(v.size)).reshape(v.shape)
