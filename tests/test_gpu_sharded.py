"""Sharded IMM on the device: pools as shards (rip_pool_skip, rip_shard_*),
summed in process and, through a one-rank NCCL group, by all_reduce.  The
seeds, theta, deltas and f must equal the single-pool IMM under the lowest-id
tie-break and the oracle's, for any number of shards."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

import ripples_b200 as rb
from oracle import oracle as O
from ripples_b200.sharded import DeviceShard, imm_sharded

pytestmark = pytest.mark.gpu


def ic_graph():
    # the 2^14-vertex IC configuration: R-MAT 2^14 / 2^18 draws, p ~ U(0, 0.1)
    return rb.HostGraph.rmat(14, 1 << 18, seed=0).with_weights(rb.WEIGHTS_UNIFORM, seed=1,
                                                               lo=0.0, hi=0.1)


def lt_graph():
    return rb.HostGraph.rmat(13, 8 << 13, seed=9).with_weights(rb.WEIGHTS_LT_NORMALIZED,
                                                               seed=109)


CASES = [("IC", ic_graph, 20, 0.5, 0), ("LT", lt_graph, 10, 0.5, 3)]


def single_pool(ctx, g, model, k, eps, seed):
    p = rb.Pool(rb.DeviceGraph(ctx, g, model))
    seeds, rec = p.imm(k, eps, 1.0, seed=seed, tiebreak=rb.TIE_LOWEST_ID)
    return seeds.tolist(), rec


@pytest.mark.parametrize("model,make,k,eps,seed", CASES, ids=["IC", "LT"])
@pytest.mark.parametrize("shards", [1, 3])
@pytest.mark.parametrize("exchange", ["sparse", "dense"])
def test_shards_equal_single_pool_and_oracle(model, make, k, eps, seed, shards, exchange):
    g = make()
    ctx = rb.Context(0)
    try:
        ref_seeds, ref = single_pool(ctx, g, model, k, eps, seed)
        dg = rb.DeviceGraph(ctx, g, model)
        sh = [DeviceShard(rb.Pool(dg)) for _ in range(shards)]
        seeds, rec = imm_sharded(sh, k, eps, 1.0, seed, exchange=exchange)
        assert seeds == ref_seeds
        assert rec["theta"] == ref.theta
        assert rec["theta_prime_deltas"] == list(ref.theta_prime_deltas[:ref.num_rounds])
        assert rec["total_sets"] == ref.total_sets
        assert rec["f"] == ref.f
        thr = O.pack(model, g.index, g.weights)
        o = O.imm(model, g.n, g.index, g.src, thr, k, eps, seed=seed, tiebreak=1)
        assert seeds == o["seeds"] and rec["theta"] == o["theta"] and rec["f"] == o["f"]
        # each shard sampled its own share: element counts add up to the pool's
        total_elems = sum(s.pool.num_elements for s in sh)
        p1 = rb.Pool(dg)
        p1.sample(rec["total_sets"], seed)
        assert total_elems == p1.num_elements
        if shards > 1:
            assert all(s.pool.num_elements < total_elems for s in sh)
    finally:
        ctx.close()


def lowest_id_max(c):
    return int(np.flatnonzero(c == c.max())[0]), int(c.max())


@pytest.mark.parametrize("n", [1 << 14, (1 << 14) - 3])
def test_shard_pick_is_lowest_id_maximum(n):
    """Picks over arbitrary summed arrays, and the chunk-maximum cache across
    decrements (apply) against a numpy restatement; n not a multiple of the
    2048-count chunk exercises the ragged last chunk."""
    import torch
    ctx = rb.Context(0)
    try:
        g = rb.HostGraph.erdos_renyi(n, 8 * n, seed=3).with_weights(rb.WEIGHTS_UNIFORM, seed=4,
                                                                    lo=0.0, hi=0.1)
        p = rb.Pool(rb.DeviceGraph(ctx, g, "IC"))
        # a pick before rip_shard_begin is refused
        t = torch.zeros(n + 4, dtype=torch.int32, device="cuda")
        with pytest.raises(rb.RipError):
            p.shard_pick(t.data_ptr())
        p.sample(100, seed=1)
        p.shard_begin(100, t.data_ptr())
        rng = np.random.default_rng(5)
        for n_max in [1, 3, 1000]:
            c = rng.integers(0, n_max, n).astype(np.uint32)
            s = torch.from_numpy(c.view(np.int32)).cuda()
            assert p.shard_pick(s.data_ptr()) == lowest_id_max(c)
        # counts above 2^31 stay unsigned
        c = np.zeros(n, np.uint32)
        c[77] = 3_000_000_000
        c[5] = 2_999_999_999
        assert p.shard_pick(torch.from_numpy(c.view(np.int32)).cuda().data_ptr()) == \
            (77, 3_000_000_000)
        # the cache: one array, decrements applied between picks
        c = rng.integers(0, 50, n).astype(np.uint32)
        s = torch.from_numpy(c.view(np.int32)).cuda()
        for step in range(30):
            assert p.shard_pick(s.data_ptr()) == lowest_id_max(c)
            v, _ = lowest_id_max(c)
            others = np.unique(rng.integers(0, n, 40))
            others = others[(c[others] > 0) & (others != v)]
            # the pick's own count to zero, then distinct others: no count below 0
            dec = np.concatenate([np.full(int(c[v]), v), others]).astype(np.uint32)
            dec = dec[:1 + step * 7]
            np.subtract.at(c, dec, 1)
            d = torch.from_numpy(dec.view(np.int32)).cuda()
            p.shard_apply(s.data_ptr(), d.data_ptr(), d.numel())
            assert np.array_equal(s.cpu().numpy().view(np.uint32), c)
        # misaligned arrays are refused
        with pytest.raises(rb.RipError):
            p.shard_pick(t.data_ptr() + 4)
        # a too short decrement list is refused before any work
        with pytest.raises(rb.RipError):
            p.shard_cover_list(0, 1, t.data_ptr(), 0)
    finally:
        ctx.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_one_rank_nccl_group_equals_single_pool():
    import torch.distributed as dist
    model, make, k, eps, seed = CASES[0]
    g = make()
    ctx = rb.Context(0)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60),
                            device_id=__import__("torch").device("cuda", 0))
    try:
        ref_seeds, ref = single_pool(ctx, g, model, k, eps, seed)
        dg = rb.DeviceGraph(ctx, g, model)
        sh = [DeviceShard(rb.Pool(dg)) for _ in range(2)]
        for exchange in ["sparse", "dense"]:
            for s in sh:
                s.pool.clear()
            seeds, rec = imm_sharded(sh, k, eps, 1.0, seed, group=dist.group.WORLD,
                                     exchange=exchange)
            assert seeds == ref_seeds and rec["theta"] == ref.theta and rec["f"] == ref.f
    finally:
        dist.destroy_process_group()
        ctx.close()
