"""Comb population control across ranks (src/AFQMC/Walkers/population_control.hpp:87-255).

Walkers are independent between combs, so a run shards its population over the GPUs of a node
(one process per GPU) and the comb is the only exchange: every rank gathers the |w| of the whole
population, runs the same comb (the walker generator is seeded identically on every rank, so all
ranks draw the same uniform as the reference's root does), computes the same deterministic
exchange plan (afqmc_plan_walker_exchange), and moves walker rows rank to rank with
point-to-point sends of packed rows (NCCL on GPUs, gloo in the CPU tests).  Slot assignment
follows swap_walkers_async (population_control.hpp:142-209): keepers stay, arrivals take the
freed slots in plan order, then the extra local copies, then the extra copies of arrivals.

The row storage is abstract (`RowStore`): `WalkerRows` moves device rows through the C ABI
(pack / unpack / copy kernels); `TensorRows` keeps rows in a plain tensor and serves the CPU
tests of the exchange logic.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from . import afqmc as A
from . import capi


class TensorRows:
    """Rows of a [n][row_len] tensor (any device)."""

    def __init__(self, t: torch.Tensor):
        self.t = t

    def __len__(self):
        return self.t.shape[0]

    def pack(self, idx):
        return self.t[torch.as_tensor(idx, dtype=torch.long, device=self.t.device)].contiguous()

    def empty(self, n):
        return torch.empty((n,) + tuple(self.t.shape[1:]), dtype=self.t.dtype, device=self.t.device)

    def unpack(self, idx, buf):
        self.t[torch.as_tensor(idx, dtype=torch.long, device=self.t.device)] = buf

    def copy(self, dst, src):
        if len(dst):
            d = torch.as_tensor(dst, dtype=torch.long, device=self.t.device)
            s = torch.as_tensor(src, dtype=torch.long, device=self.t.device)
            self.t[d] = self.t[s]


class WalkerRows:
    """Walker-buffer rows of a WalkerSet, moved by the library's pack / unpack / copy kernels."""

    def __init__(self, wset: A.WalkerSet):
        self.ws = wset

    def __len__(self):
        return self.ws.W

    def _idx(self, idx):
        return torch.as_tensor(np.asarray(idx, dtype=np.int32), device=self.ws.buffer.device)

    def pack(self, idx):
        return self.ws.pack_rows(self._idx(idx))

    def empty(self, n):
        return torch.empty((n, self.ws.walker_size), dtype=torch.complex128,
                           device=self.ws.buffer.device)

    def unpack(self, idx, buf):
        self.ws.unpack_rows(self._idx(idx), buf)

    def copy(self, dst, src):
        if len(dst):
            self.ws.copy_rows(self._idx(dst), self._idx(src))


def _p2p(ops):
    """Posts point-to-point ops in order and waits for all of them.  Under a backend without
    device point-to-point (gloo) device tensors are staged through host memory: a send copies
    the packed rows to the host, a receive lands in a host buffer copied to the device after."""
    if not ops:
        return
    stage = dist.get_backend() != "nccl"
    reqs, landed = [], []
    for op, t, peer in ops:
        buf = t
        if stage and t.is_cuda:
            if op == "send":
                buf = t.cpu()
            else:
                buf = torch.empty(t.shape, dtype=t.dtype)
                landed.append((t, buf))
        reqs.append((dist.isend if op == "send" else dist.irecv)(buf, peer))
    for r in reqs:
        r.wait()
    for t, buf in landed:
        t.copy_(buf)


def exchange_walkers(rows, offspring, counts, rank):
    """swap_walkers_async (population_control.hpp:142-209) over torch.distributed point-to-point.

    offspring: copies of every walker of the global population, rank-major; counts: walkers per
    rank.  Collective over the default process group (every rank calls it with the same
    offspring and counts).  Returns the global source index of every local slot."""
    offspring = np.asarray(offspring, dtype=np.int32)
    counts = [int(c) for c in counts]
    nw = counts[rank]
    if len(rows) != nw:
        raise ValueError(f"exchange_walkers: {len(rows)} rows, but rank {rank} holds {nw}")
    plan = A.plan_walker_exchange(offspring, np.asarray(counts, dtype=np.int32))
    first = int(sum(counts[:rank]))
    keep = [int(x) for x in offspring[first:first + nw]]
    for src, wk, dst, copies in plan:
        if src == rank:
            keep[wk] -= copies
    src_of = list(range(first, first + nw))
    free = [i for i in range(nw) if keep[i] == 0]
    nxt = 0
    # one message per (source, destination) pair: the rows in plan order
    sends, recvs = {}, {}
    arrivals = []
    for src, wk, dst, copies in plan:
        if src == rank:
            sends.setdefault(dst, []).append(wk)
        elif dst == rank:
            slot = free[nxt]
            nxt += 1
            recvs.setdefault(src, []).append(slot)
            arrivals.append((slot, copies))
            src_of[slot] = int(sum(counts[:src])) + wk
    ops, inbox = [], {}
    for dst in sorted(sends):
        ops.append(("send", rows.pack(sends[dst]), dst))
    for src in sorted(recvs):
        inbox[src] = rows.empty(len(recvs[src]))
        ops.append(("recv", inbox[src], src))
    _p2p(ops)
    for src, slots in recvs.items():
        rows.unpack(slots, inbox[src])
    # extra local copies, then extra copies of the arrivals, into the remaining freed slots
    dst_l, src_l = [], []
    for i in range(nw):
        for _ in range(1, keep[i]):
            dst_l.append(free[nxt])
            src_l.append(i)
            src_of[free[nxt]] = first + i
            nxt += 1
    for slot, copies in arrivals:
        for _ in range(1, copies):
            dst_l.append(free[nxt])
            src_l.append(slot)
            src_of[free[nxt]] = src_of[slot]
            nxt += 1
    if nxt != len(free):
        raise ValueError(f"exchange_walkers: {len(free) - nxt} slots left unfilled")
    # copies read only kept or arrived rows, never a freed slot that is itself a copy target
    rows.copy(dst_l, src_l)
    return np.asarray(src_of)


def _all_gather_varlen(x: np.ndarray, device):
    """Every rank's 1-D array, concatenated in rank order."""
    world = dist.get_world_size()
    n = torch.tensor([x.size], dtype=torch.int64, device=device)
    ns = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(ns, n)
    ns = [int(v.item()) for v in ns]
    mx = max(ns)
    buf = torch.zeros(mx, dtype=torch.float64, device=device)
    buf[:x.size] = torch.as_tensor(x, dtype=torch.float64, device=device)
    outs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(outs, buf)
    return np.concatenate([o[:k].cpu().numpy() for o, k in zip(outs, ns)]), ns


def population_control_distributed(wset: A.WalkerSet, rng: A.HostRandomGenerator):
    """population_control (population_control.hpp:218-255) over the default process group:
    gather |w|, comb (identical on every rank), exchange rows, w <- w/|w|.  Returns the
    offspring of the global population."""
    device = wset.buffer.device if dist.get_backend() == "nccl" else "cpu"
    w = np.abs(wset.getProperty(capi.WEIGHT))
    all_w, counts = _all_gather_varlen(w, device)
    offspring = A.comb(rng, all_w, int(sum(counts)))
    exchange_walkers(WalkerRows(wset), offspring, counts, dist.get_rank())
    wset.normalize_weights()
    return offspring
