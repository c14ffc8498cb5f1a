"""The distributed comb over the library's walker rows (population_control_distributed with
WalkerRows: the afqmc_wset_pack_rows / unpack_rows / copy_rows kernels) in two processes that
share one GPU, over a gloo process group (rows staged through host memory; no kernel of one
process waits on the other).  Every rank's walker rows after the comb are checked against the
oracle's slot map of swap_walkers_async (population_control.hpp:142-209)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import afqmc as O

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _weights(counts, seed):
    rs = np.random.default_rng(seed)
    w_all = rs.random(sum(counts)) + 0.05
    w_all[rs.random(sum(counts)) < 0.3] = 0.0
    w_all[0] = max(w_all[0], 0.5)
    w_all[:counts[0]] *= 3.0  # heavier on rank 0: walkers have to move between the ranks
    return w_all


def _worker(rank, world, port, counts, seed, result_dir):
    from datetime import timedelta

    from safire_b200 import afqmc as A
    from safire_b200.population import population_control_distributed
    from safire_b200.synth import make_workload
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        wl = make_workload("cfg1", W=counts[rank], M=16, N=4, Nc=16)
        ham = A.HamiltonianOperations(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij,
                                      wl.E0, wl.PsiT)
        ws = A.WalkerSet(wl.walker_type, wl.M, wl.nup, wl.ndn, counts[rank])
        ws.init_from_trial(ham)
        first = sum(counts[:rank])
        w_all = _weights(counts, seed)
        nrow = ws.walker_size
        # every row identifiable by its global walker index g: element c holds g + i c
        g = torch.arange(first, first + counts[rank], dtype=torch.float64, device="cuda")
        c = torch.arange(nrow, dtype=torch.float64, device="cuda")
        ws.buffer.copy_(torch.complex(g[:, None].expand(-1, nrow), c[None, :].expand(len(g), -1)))
        torch.cuda.synchronize()
        ws.setProperty(A.capi.WEIGHT, w_all[first:first + counts[rank]].astype(complex))
        rng = A.HostRandomGenerator(A.split_seed(seed, 0, 0))
        off = population_control_distributed(ws, rng)
        torch.cuda.synchronize()
        ref_off = O.comb(O.HostRandomGenerator(O.split_seed(seed, 0, 0)), w_all, sum(counts))
        assert np.array_equal(off, ref_off)
        src = O.swap_walkers_slot_map(ref_off, counts, rank)
        buf = ws.buffer.cpu().numpy()
        prop0 = ws.prop0
        for slot, gsrc in enumerate(src):
            row = buf[slot]
            assert np.all(row[:prop0].real == gsrc), (rank, slot, gsrc)
            assert np.all(row[:prop0].imag == np.arange(prop0)), (rank, slot)
            # the weight column holds w / |w| after the comb
            assert abs(row[prop0 + A.capi.WEIGHT] - 1.0) < 1e-15, (rank, slot)
        with open(os.path.join(result_dir, f"rank{rank}.ok"), "w") as f:
            f.write(str(len(src)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("counts,seed", [([6, 10], 3), ([9, 9], 4)])
def test_walker_rows_distributed_comb(cuda, tmp_path, counts, seed):
    w_all = _weights(counts, seed)
    off = O.comb(O.HostRandomGenerator(O.split_seed(seed, 0, 0)), w_all, sum(counts))
    assert len(O.plan_walker_exchange(off, counts)) > 0  # rows do move between the ranks
    mp.spawn(_worker, args=(len(counts), _free_port(), counts, seed, str(tmp_path)),
             nprocs=len(counts), join=True)
    for r in range(len(counts)):
        assert (tmp_path / f"rank{r}.ok").exists()
