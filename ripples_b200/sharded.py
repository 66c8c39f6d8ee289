"""Sharded IMM: the RRR sets of one query split across shards -- one pool per
GPU, one process per GPU over ``torch.distributed`` (NCCL), and optionally
several pools per process -- with the shards' vertex counts combined at
every pick.

Reference: the MPI IMM (include/ripples/mpi/imm.h:150-250: every rank samples
its share of theta, f is taken over all ranks' sets) and its
FindMostInfluentialSet (include/ripples/mpi/find_most_influential.h:449-690:
per pick, the ranks' vertex counters are reduced, the maximum is picked and
every rank updates the counters of its own sets).

The union of the shards' sets is exactly the sets 0 .. S-1 one pool holds:
each growth of the pool from S_old to S_new sets is cut into contiguous id
ranges, one per shard in (rank, local shard) order; a shard samples its own
range and appends empty placeholders for the other shards' ids
(``rip_pool_skip``), so set ids, and with them the sets, are the single-pool
ones.  The picks are the largest summed count, the lowest vertex id among
equal counts -- the reference's GPU pick over the reduced counters
(thrust::max_element, mpi/find_most_influential.h:505-511) and this library's
``TIE_LOWEST_ID``.  So seeds, theta, the per-round theta' deltas and f equal
``Pool.imm(..., tiebreak=TIE_LOWEST_ID)`` on one device whatever the number
of shards.  (The reference's MPI IMM instead samples theta/ranks + 1 sets per
rank from rank-specific streams, so its answer moves with the rank count.)

Counts are summed once per selection (an in-process sum over the local
shards, then ``all_reduce`` over ``group``); after each pick the shards
exchange either
- ``"sparse"``: the members of the sets each shard newly covered,
  gathered from every shard (``all_gather``) and subtracted from the
  replicated sums, whose pick recomputes only the 2048-count chunks they
  touched -- the bytes exchanged are the decrements, not n counts; or
- ``"dense"``: every shard's updated counts, summed again as at the start
  (n counts per pick, as the reference's MPI_Reduce of its counter array).
Both give the same picks.  ``"auto"`` (default) takes sparse whenever there
is something to exchange (a group, or several local shards) and dense for a
single shard alone, where the sum is its own counts (on one B200 at 2^24
that saves a host synchronisation a pick: 63 against 73 ms of selection per
IMM).

A shard is any object with ``n``, ``num_sets``, ``grow(seed, skip_before,
count, skip_after)``, ``begin(num_sets) -> counts``, ``cover(vertex, gain) ->
counts``, ``cover_list(vertex, gain) -> decrements``, ``apply(total,
decrements)`` and ``pick(total) -> (vertex, gain)``; ``counts`` and
``total`` are int32 tensors of n entries holding uint32 bits, decrements an
int32 tensor of vertex ids.  :class:`DeviceShard` is the library's.
"""
from __future__ import annotations

import math
import time
from typing import List, Optional, Sequence, Tuple

from . import _lib


class DeviceShard:
    """One pool on one GPU as a shard.  Its counts live in a torch int32
    tensor on the pool's device (uint32 bits: sums wrap like uint32, and the
    true sums stay below 2^32 because a selection has fewer than 2^32 sets)."""

    def __init__(self, pool):
        import torch
        self.pool = pool
        self.n = pool.graph.n
        self.device = torch.device("cuda", pool.ctx.device)
        # rip_shard_* want 16-byte aligned arrays; torch allocations are
        self.counts = torch.zeros(self.n, dtype=torch.int32, device=self.device)
        self.dec = torch.zeros(4, dtype=torch.int32, device=self.device)

    @property
    def num_sets(self) -> int:
        return self.pool.num_sets

    def grow(self, seed: int, skip_before: int, count: int, skip_after: int) -> None:
        self.pool.skip(skip_before)
        self.pool.sample(count, seed)
        self.pool.skip(skip_after)

    def begin(self, num_sets: int):
        import torch
        elements = self.pool.shard_begin(num_sets, self.counts.data_ptr())
        if self.dec.numel() < elements:
            self.dec = torch.empty(elements, dtype=torch.int32, device=self.device)
        return self.counts

    def cover(self, vertex: int, gain: int):
        self.pool.shard_cover(vertex, gain, self.counts.data_ptr())
        return self.counts

    def cover_list(self, vertex: int, gain: int):
        m = self.pool.shard_cover_list(vertex, gain, self.dec.data_ptr(), self.dec.numel())
        return self.dec[:m]

    def apply(self, total, dec) -> None:
        assert total.device == self.device and dec.device == self.device
        dec = dec.contiguous()
        self.pool.shard_apply(total.data_ptr(), dec.data_ptr() if dec.numel() else None,
                              dec.numel())

    def pick(self, total) -> Tuple[int, int]:
        assert total.device == self.device and total.dtype.itemsize == 4
        return self.pool.shard_pick(total.data_ptr())


def split(first: int, last: int, shards: int, index: int) -> Tuple[int, int]:
    """Shard ``index``'s contiguous id range of the growth [first, last)."""
    d = last - first
    return first + d * index // shards, first + d * (index + 1) // shards


class ShardedSelection:
    """Greedy lowest-id max coverage over the shards' sets [0, num_sets)."""

    def __init__(self, shards: Sequence, group=None, exchange: str = "auto"):
        if exchange not in ("auto", "sparse", "dense"):
            raise ValueError("exchange: 'auto', 'sparse' or 'dense'")
        if exchange == "auto":  # one shard alone has nothing to exchange
            exchange = "sparse" if group is not None or len(shards) > 1 else "dense"
        self.shards = list(shards)
        self.group = group
        self.exchange = exchange
        self._total = None
        self.allreduce_ms = 0.0  # host ms in collectives (sums and gathers)
        self.exchanged = 0  # decrement entries this rank received, padding included
        self.picks = 0

    def _sum(self, parts):
        import torch
        import torch.distributed as dist
        if len(parts) == 1:
            total = parts[0]  # the shard rewrites it with its own counts before the next sum
        else:
            if self._total is None or self._total.shape != parts[0].shape:
                self._total = torch.empty_like(parts[0])
            total = self._total
            total.copy_(parts[0])
            for p in parts[1:]:
                total.add_(p.to(total.device))
        if self.group is not None:
            t0 = time.perf_counter()
            dist.all_reduce(total, group=self.group)
            if total.is_cuda:
                torch.cuda.current_stream(total.device).synchronize()
            self.allreduce_ms += (time.perf_counter() - t0) * 1e3
        elif total.is_cuda:
            torch.cuda.current_stream(total.device).synchronize()
        return total

    def _gather(self, parts):
        """Every shard's decrement list, on the first shard's device."""
        import torch
        import torch.distributed as dist
        local = parts[0] if len(parts) == 1 else torch.cat([p.to(parts[0].device)
                                                            for p in parts])
        if self.group is None:
            return local
        t0 = time.perf_counter()
        world = dist.get_world_size(self.group)
        size = torch.tensor([local.numel()], dtype=torch.int64, device=local.device)
        sizes = [torch.empty_like(size) for _ in range(world)]
        dist.all_gather(sizes, size, group=self.group)
        sizes = [int(x.item()) for x in sizes]
        longest = max(sizes)
        if longest == 0:
            out = local[:0]
        else:
            buf = torch.empty(longest, dtype=local.dtype, device=local.device)
            buf[:local.numel()].copy_(local)
            recv = [torch.empty_like(buf) for _ in range(world)]
            dist.all_gather(recv, buf, group=self.group)
            out = torch.cat([r[:m] for r, m in zip(recv, sizes)])
            self.exchanged += world * longest
        if out.is_cuda:
            torch.cuda.current_stream(out.device).synchronize()
        self.allreduce_ms += (time.perf_counter() - t0) * 1e3
        return out

    def select(self, num_sets: int, k: int) -> Tuple[List[int], List[int], float]:
        """(seeds, gains, f) with f = covered / num_sets."""
        total = self._sum([s.begin(num_sets) for s in self.shards])
        seeds: List[int] = []
        gains: List[int] = []
        covered = 0
        while len(seeds) < k:
            v, gain = self.shards[0].pick(total)
            self.picks += 1
            if gain == 0:
                break
            seeds.append(v)
            gains.append(gain)
            covered += gain
            if len(seeds) == k or covered == num_sets:
                break
            if self.exchange == "dense":
                total = self._sum([s.cover(v, gain) for s in self.shards])
            else:
                dec = self._gather([s.cover_list(v, gain) for s in self.shards])
                self.shards[0].apply(total, dec)
        f = covered / num_sets if num_sets else 0.0
        return seeds, gains, f


def imm_sharded(shards: Sequence, k: int, epsilon: float, l: float = 1.0, seed: int = 0,
                group=None, exchange: str = "auto") -> Tuple[List[int], dict]:
    """IMM over sharded pools; returns (seeds, record).

    ``shards`` are this process's shards; ``group`` the process group over
    which every process runs the same call with its own shards (None: one
    process).  The martingale rounds follow include/ripples/imm.h:145-260 and
    the final selection imm.h:836-850, with theta' / theta from the library's
    restatement of imm.h:77-128."""
    if group is not None:
        import torch.distributed as dist
        rank, world = dist.get_rank(group), dist.get_world_size(group)
    else:
        rank, world = 0, 1
    shards = list(shards)
    if not shards or not epsilon > 0:
        raise ValueError("imm_sharded: at least one shard and epsilon > 0")
    local = len(shards)
    total_shards = world * local
    n = shards[0].n
    S = shards[0].num_sets
    if any(s.num_sets != S or s.n != n for s in shards):
        raise ValueError("imm_sharded: shards must hold the same graph and set count")
    sel = ShardedSelection(shards, group, exchange)
    L = _lib.lib
    rec = {"theta_prime_deltas": [], "round_generate_ms": [], "round_select_ms": []}
    t_total = time.perf_counter()

    def grow(to: int) -> None:
        nonlocal S
        for j, sh in enumerate(shards):
            a, b = split(S, to, total_shards, rank * local + j)
            sh.grow(seed, a - S, b - a, to - b)
        S = to

    l = l * (1 + 1 / math.log2(n))
    eps_prime = math.sqrt(2) * epsilon
    LB = 0.0
    x = 1
    if S != 0:
        x = int(L.rip_inv_theta_prime(S // 2, eps_prime, l, k, n))
    t_est = time.perf_counter()
    while x < math.log2(n):
        theta_prime = int(L.rip_theta_prime(x, eps_prime, l, k, n))
        t0 = time.perf_counter()
        delta = 0
        if max(theta_prime, 0) > S:
            delta = theta_prime - S
            grow(theta_prime)
        gen_ms = (time.perf_counter() - t0) * 1e3
        t0 = time.perf_counter()
        _, _, f = sel.select(S, k)
        rec["theta_prime_deltas"].append(delta)
        rec["round_generate_ms"].append(gen_ms)
        rec["round_select_ms"].append((time.perf_counter() - t0) * 1e3)
        if f >= 2.0 ** -x:
            LB = (n * f) / (1 + eps_prime)
            break
        x += 1
    theta = int(L.rip_theta(epsilon, l, k, LB, n))
    rec["theta_estimation_ms"] = (time.perf_counter() - t_est) * 1e3
    rec["theta"] = theta
    t0 = time.perf_counter()
    if theta > S:
        grow(theta)
    rec["generate_ms"] = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    seeds, gains, f = sel.select(min(theta, S), k)
    rec["select_ms"] = (time.perf_counter() - t0) * 1e3
    rec.update(f=f, total_sets=S, gains=gains, shards=total_shards, picks=sel.picks,
               allreduce_ms=sel.allreduce_ms, exchange=sel.exchange, exchanged=sel.exchanged,
               total_ms=(time.perf_counter() - t_total) * 1e3)
    return seeds, rec
