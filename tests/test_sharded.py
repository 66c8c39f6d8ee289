"""The sharded IMM's host logic on CPU: set-id ranges, the per-pick sum over
local shards and gloo ranks, and the martingale around them.  The shards
here hold the oracle's sets on the host (test infrastructure standing in for
the device pools); the answer must equal the oracle's single-pool IMM under
the lowest-id tie-break, whatever the number of ranks and shards."""
import os
import socket
import sys
from datetime import timedelta

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class OracleShard:
    """A shard whose sets come from the oracle, counted and covered with
    numpy.  Ids of other shards are empty placeholders, as on the device."""

    def __init__(self, model, g, thr):
        self.model, self.g, self.thr = model, g, thr
        self.n = g.n
        self.off = [np.zeros(1, np.uint64)]  # per growth: CSR pieces
        self.lens = []                       # per set id: its length (0 = not ours)
        self.vtx = []

    @property
    def num_sets(self):
        return len(self.lens)

    def grow(self, seed, skip_before, count, skip_after):
        from oracle import oracle as O
        self.lens += [0] * skip_before
        if count:
            off, vtx, _ = O.sample(self.model, self.n, self.g.index, self.g.src, self.thr, seed,
                                   len(self.lens), count)
            self.lens += np.diff(off).astype(np.int64).tolist()
            self.vtx.append(vtx)
        self.lens += [0] * skip_after

    def begin(self, num_sets):
        import torch
        lens = np.asarray(self.lens[:num_sets], dtype=np.int64)
        vtx = np.concatenate(self.vtx) if self.vtx else np.zeros(0, np.uint32)
        vtx = vtx[:lens.sum()]
        self.set_of = np.repeat(np.arange(num_sets), lens)
        self.members = vtx.astype(np.int64)
        self.start = np.concatenate([[0], np.cumsum(lens)])
        self.covered = np.zeros(num_sets, bool)
        self.cnt = np.bincount(self.members, minlength=self.n).astype(np.int64)
        return torch.from_numpy(self.cnt.astype(np.int32))

    def _cover(self, v):
        sets = np.unique(self.set_of[self.members == v])
        sets = sets[~self.covered[sets]]
        self.covered[sets] = True
        dec = [self.members[self.start[s]:self.start[s + 1]] for s in sets]
        return np.concatenate(dec) if dec else np.zeros(0, np.int64)

    def cover(self, v, gain):
        import torch
        np.subtract.at(self.cnt, self._cover(v), 1)
        return torch.from_numpy(self.cnt.astype(np.int32))

    def cover_list(self, v, gain):
        import torch
        return torch.from_numpy(self._cover(v).astype(np.int32))

    def apply(self, total, dec):
        t = total.numpy()  # shares the tensor's memory
        np.subtract.at(t, dec.numpy(), 1)

    def pick(self, total):
        t = total.numpy().view(np.uint32)
        v = int(np.argmax(t))  # first maximum: the lowest id
        return v, int(t[v])


def graph(model):
    import ripples_b200 as rb
    if model == "IC":
        return rb.HostGraph.rmat(10, 8 << 10, seed=21).with_weights(rb.WEIGHTS_UNIFORM, seed=22,
                                                                    lo=0.0, hi=0.2)
    return rb.HostGraph.rmat(10, 8 << 10, seed=23).with_weights(rb.WEIGHTS_LT_NORMALIZED,
                                                                seed=24)


QUERY = dict(k=8, epsilon=0.5, seed=7)


def oracle_answer(model, g):
    from oracle import oracle as O
    thr = O.pack(model, g.index, g.weights)
    return O.imm(model, g.n, g.index, g.src, thr, QUERY["k"], QUERY["epsilon"],
                 seed=QUERY["seed"], tiebreak=1)


def run_sharded(model, g, local, group=None, exchange="sparse"):
    from oracle import oracle as O
    from ripples_b200.sharded import imm_sharded
    thr = O.pack(model, g.index, g.weights)
    shards = [OracleShard(model, g, thr) for _ in range(local)]
    seeds, rec = imm_sharded(shards, QUERY["k"], QUERY["epsilon"], 1.0, QUERY["seed"], group,
                             exchange)
    return seeds, rec, shards


def test_split_ranges_tile_each_growth():
    from ripples_b200.sharded import split
    for first, last, shards in [(0, 10, 3), (7, 8, 4), (5, 5, 2), (100, 1234, 8)]:
        got = [split(first, last, shards, i) for i in range(shards)]
        assert got[0][0] == first and got[-1][1] == last
        for (a, b), (c, d) in zip(got, got[1:]):
            assert b == c and a <= b
        assert sum(b - a for a, b in got) == last - first


@pytest.mark.parametrize("model", ["IC", "LT"])
@pytest.mark.parametrize("local", [1, 3])
@pytest.mark.parametrize("exchange", ["sparse", "dense"])
def test_one_process_shards_equal_single_pool(model, local, exchange):
    g = graph(model)
    seeds, rec, shards = run_sharded(model, g, local, exchange=exchange)
    o = oracle_answer(model, g)
    assert seeds == o["seeds"]
    assert rec["theta"] == o["theta"]
    assert [d for d in rec["theta_prime_deltas"]] == o["deltas"]
    assert rec["total_sets"] == o["total_sets"]
    assert rec["f"] == pytest.approx(o["f"], abs=0, rel=0)
    # every shard sampled a share; together they hold each id once
    owned = np.array([[l > 0 for l in s.lens] for s in shards])
    if local > 1:
        assert (owned.sum(axis=1) > 0).all()
        assert owned.sum(axis=0).max() == 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, model, local, exchange, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        g = graph(model)
        seeds, rec, shards = run_sharded(model, g, local, group=dist.group.WORLD,
                                         exchange=exchange)
        owned = [int(sum(l > 0 for l in s.lens)) for s in shards]
        out.put((rank, seeds, rec["theta"], rec["theta_prime_deltas"], rec["f"],
                 rec["total_sets"], owned, rec["exchanged"]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("model,local,exchange", [("IC", 2, "sparse"), ("LT", 1, "sparse"),
                                                  ("IC", 1, "dense")])
def test_two_gloo_ranks_equal_single_pool(model, local, exchange):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, model, local, exchange, out))
             for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    o = oracle_answer(model, graph(model))
    for _, seeds, theta, deltas, f, total, owned, exchanged in res:
        assert seeds == o["seeds"]
        assert theta == o["theta"] and deltas == o["deltas"] and total == o["total_sets"]
        assert f == o["f"]
        # sparse: decrement lists crossed between the ranks; dense: none
        assert (exchanged > 0) == (exchange == "sparse")
    # the ranks sampled disjoint shares that add up to every set
    assert sum(sum(r[6]) for r in res) == o["total_sets"]
    assert all(min(r[6]) > 0 for r in res)
