"""Comb population control across ranks: the exchange of walker rows (swap_walkers_async,
population_control.hpp:142-209) run as gloo ranks on the CPU, checked slot by slot against the
oracle's restatement, and the full gather -> comb -> exchange sequence checked against the
single-process comb of the concatenated population."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import afqmc as O


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))


def _rows(counts, rank):
    first = sum(counts[:rank])
    ids = torch.arange(first, first + counts[rank], dtype=torch.float64)
    # a few columns per row so that whole rows are checked, not one number
    return torch.stack([ids, 10 * ids + 1, -ids], dim=1).contiguous()


def _exchange_worker(rank, world, port, counts, offspring):
    from safire_b200.population import TensorRows, exchange_walkers
    _init(rank, world, port)
    try:
        rows = TensorRows(_rows(counts, rank))
        src = exchange_walkers(rows, offspring, counts, rank)
        ref = O.swap_walkers_slot_map(offspring, counts, rank)
        assert np.array_equal(src, ref), (rank, src, ref)
        got = rows.t.numpy()
        assert np.array_equal(got[:, 0], ref.astype(np.float64)), (rank, got[:, 0], ref)
        assert np.array_equal(got[:, 1], 10 * ref + 1.0)
        assert np.array_equal(got[:, 2], -ref.astype(np.float64))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _random_offspring(rs, counts):
    # a population-preserving offspring vector: comb of random weights (zeros included), heavier
    # on rank 0 so that walkers have to move between ranks
    ntot = sum(counts)
    w = rs.random(ntot)
    w[:counts[0]] *= 4.0
    w[rs.random(ntot) < 0.3] = 0.0
    w[0] = max(w[0], 0.1)
    return O.comb(O.HostRandomGenerator(int(rs.integers(1 << 30))), w, ntot)


@pytest.mark.parametrize("counts,seed", [([5, 7], 0), ([8, 8], 1), ([4, 6, 3], 2),
                                         ([2, 9, 2], 3), ([6, 0, 5], 4)])
def test_exchange_walkers_gloo(counts, seed):
    rs = np.random.default_rng(seed)
    offspring = _random_offspring(rs, counts)
    # the exchange has to move walkers for the test to mean something
    plan = O.plan_walker_exchange(offspring, counts)
    assert len(plan) > 0
    mp.spawn(_exchange_worker, args=(len(counts), _free_port(), counts, offspring),
             nprocs=len(counts), join=True)


def test_exchange_walkers_no_transfer():
    """Every rank already holds its share: the exchange is local copies only."""
    counts = [4, 4]
    offspring = np.array([2, 0, 1, 1, 1, 1, 0, 2], dtype=np.int32)
    assert O.plan_walker_exchange(offspring, counts) == []
    mp.spawn(_exchange_worker, args=(2, _free_port(), counts, offspring), nprocs=2, join=True)


def _comb_worker(rank, world, port, counts, seed):
    from safire_b200 import afqmc as A
    from safire_b200.population import TensorRows, _all_gather_varlen, exchange_walkers
    _init(rank, world, port)
    try:
        rs = np.random.default_rng(seed)
        w_all = rs.random(sum(counts)) + 0.05
        first = sum(counts[:rank])
        w_local = w_all[first:first + counts[rank]]
        gathered, ns = _all_gather_varlen(w_local, "cpu")
        assert ns == counts and np.array_equal(gathered, w_all)
        # every rank combs with an identically seeded generator
        rng = A.HostRandomGenerator(A.split_seed(seed, 0, 0))
        off = A.comb(rng, gathered, sum(counts))
        ref = O.comb(O.HostRandomGenerator(O.split_seed(seed, 0, 0)), w_all, sum(counts))
        assert np.array_equal(off, ref)
        rows = TensorRows(_rows(counts, rank))
        src = exchange_walkers(rows, off, counts, rank)
        assert np.array_equal(src, O.swap_walkers_slot_map(ref, counts, rank))
        # the union over ranks holds every walker exactly offspring times
        cnt = torch.zeros(sum(counts), dtype=torch.int64)
        for g in src:
            cnt[int(g)] += 1
        dist.all_reduce(cnt)
        assert np.array_equal(cnt.numpy(), ref)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("counts,seed", [([16, 16], 11), ([10, 13, 7], 12)])
def test_distributed_comb_matches_single_process(counts, seed):
    mp.spawn(_comb_worker, args=(len(counts), _free_port(), counts, seed), nprocs=len(counts),
             join=True)
