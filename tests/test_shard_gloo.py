"""Multi-rank sample sharding on CPU: two gloo ranks each run the oracle's
recurrence (or transport) on their block of global sample columns and one
all-reduce forms the result, which must equal the single-process oracle on
all columns (the GPU path uses the same rsatb_b200.shard logic over NCCL)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

import oracle
from rsatb_b200 import lattice
from rsatb_b200.shard import combine_average, sample_block

WORLD = 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _samples(H, first, count, seed=20240917):
    n_atoms = H.n_rows
    return oracle.set_random(seed, 0, True, np.arange(n_atoms), 1, H.n_rows, count, True,
                             first_column=first)


def _kpm_rank(rank, port, R_total, out):
    import torch.distributed as dist
    from rsatb_b200.shard import torch_all_reduce_sum
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    try:
        H, _, _ = lattice.graphene(6, 6)
        op = oracle.make_op(oracle.Bsr(H.n_block_rows, H.n_block_rows, 1, H.row_ptr, H.col_ind,
                                       H.values), 0.0, 9.0)
        first, count = sample_block(R_total, WORLD, rank)
        mu = oracle.kpm_moments(op, _samples(H, first, count), 24)
        mu = combine_average(mu, count, torch_all_reduce_sum(), R_total)
        if rank == 0:
            np.save(out, mu)
    finally:
        dist.destroy_process_group()


def test_sample_block_partition():
    for n in (1, 5, 8, 17):
        for w in (1, 2, 3, 4):
            blocks = [sample_block(n, w, r) for r in range(w)]
            cols = [c for f, k in blocks for c in range(f, f + k)]
            assert cols == list(range(n))


@pytest.mark.parametrize("R_total", [4, 5])
def test_two_gloo_ranks_equal_single_process_kpm(tmp_path, R_total):
    import torch.multiprocessing as mp
    out = str(tmp_path / "mu.npy")
    mp.start_processes(_kpm_rank, args=(_free_port(), R_total, out), nprocs=WORLD,
                       start_method="spawn")
    mu_sharded = np.load(out)
    H, _, _ = lattice.graphene(6, 6)
    op = oracle.make_op(oracle.Bsr(H.n_block_rows, H.n_block_rows, 1, H.row_ptr, H.col_ind,
                                   H.values), 0.0, 9.0)
    mu_all = oracle.kpm_moments(op, _samples(H, 0, R_total), 24)
    assert np.abs(mu_sharded - mu_all).max() < 1e-13


def _transport_rank(rank, port, out):
    import torch.distributed as dist
    from rsatb_b200.shard import torch_all_reduce_sum
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    try:
        H, _, _, disp = lattice.twisted_bilayer_graphene(m=1, tiles=(3, 3))
        V = [oracle.Bsr(v.n_block_rows, v.n_block_rows, 1, v.row_ptr, v.col_ind, v.values,
                        imag=True) for v in lattice.commutator_velocity(H, disp)]
        op = oracle.make_op(oracle.Bsr(H.n_block_rows, H.n_block_rows, 1, H.row_ptr, H.col_ind,
                                       H.values), -1.0, 10.0)
        first, count = sample_block(4, WORLD, rank)
        sig, _ = oracle.fftcheb(op, V, _samples(H, first, count), 16)
        sig = combine_average(sig, count, torch_all_reduce_sum(), 4)
        if rank == 0:
            np.save(out, sig)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_equal_single_process_transport(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "sig.npy")
    mp.start_processes(_transport_rank, args=(_free_port(), out), nprocs=WORLD,
                       start_method="spawn")
    H, _, _, disp = lattice.twisted_bilayer_graphene(m=1, tiles=(3, 3))
    V = [oracle.Bsr(v.n_block_rows, v.n_block_rows, 1, v.row_ptr, v.col_ind, v.values,
                    imag=True) for v in lattice.commutator_velocity(H, disp)]
    op = oracle.make_op(oracle.Bsr(H.n_block_rows, H.n_block_rows, 1, H.row_ptr, H.col_ind,
                                   H.values), -1.0, 10.0)
    sig_all, _ = oracle.fftcheb(op, V, _samples(H, 0, 4), 16)
    assert np.abs(np.load(out) - sig_all).max() <= 1e-12 * np.abs(sig_all).max()


def test_partition_kpoints_matches_reference_rules():
    """kpoint_partition.hpp's tests (test_setup_stages.cpp:40-93): one rank
    owns everything; every k-point has exactly one colour and ranks of a
    colour agree; npar above the world size is clamped; a rank outside the
    communicator is refused."""
    from rsatb_b200.shard import kpoint_colour, partition_kpoints
    ks = [[0.1 * i, 0.0, 0.0] for i in range(7)]
    assert [i for i, _ in partition_kpoints(ks[:5], 1, 0, 1)] == [0, 1, 2, 3, 4]
    for ws in (1, 2, 3, 4, 8):
        for npar in range(1, ws + 1):
            per_colour, covered = {}, set()
            for r in range(ws):
                idx = [i for i, _ in partition_kpoints(ks, npar, r, ws)]
                c = kpoint_colour(npar, r, ws)
                per_colour.setdefault(c, idx)
                assert per_colour[c] == idx
                covered.update(idx)
            assert covered == set(range(7))
    assert {i for r in range(2) for i, _ in partition_kpoints(ks[:4], 16, r, 2)} == set(range(4))
    with pytest.raises(ValueError):
        partition_kpoints(ks[:2], 1, 4, 4)
    with pytest.raises(ValueError):
        partition_kpoints(ks[:2], 1, 0, 0)


def _kpoint_rank(rank, port, world, npar, out):
    import torch.distributed as dist
    from rsatb_b200.shard import gather_kpoint_results, partition_kpoints, torch_all_reduce_sum
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ks = [[0.05 * i, 0.02 * i, 0.0] for i in range(5)]
        local = np.zeros((5, 3))
        for i, k in partition_kpoints(ks, npar, rank, world):
            local[i] = [i, k[0], k[1]]     # any per-k-point result
        full = gather_kpoint_results(local, npar, rank, world, torch_all_reduce_sum())
        np.save(out + f".{rank}.npy", full)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,npar", [(2, 2), (3, 3), (3, 2), (2, 1)])
def test_gather_kpoint_results_gloo(tmp_path, world, npar):
    """Every rank receives the full per-k-point array, each k-point counted
    once although several ranks of a colour computed it."""
    import torch.multiprocessing as mp
    out = str(tmp_path / "k")
    mp.start_processes(_kpoint_rank, args=(_free_port(), world, npar, out), nprocs=world,
                       start_method="spawn")
    want = np.array([[i, 0.05 * i, 0.02 * i] for i in range(5)])
    for r in range(world):
        assert np.abs(np.load(out + f".{r}.npy") - want).max() < 1e-15
