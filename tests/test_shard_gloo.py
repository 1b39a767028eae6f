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
