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
def test_shards_equal_single_pool_and_oracle(model, make, k, eps, seed, shards):
    g = make()
    ctx = rb.Context(0)
    try:
        ref_seeds, ref = single_pool(ctx, g, model, k, eps, seed)
        dg = rb.DeviceGraph(ctx, g, model)
        sh = [DeviceShard(rb.Pool(dg)) for _ in range(shards)]
        seeds, rec = imm_sharded(sh, k, eps, 1.0, seed)
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


def test_shard_pick_is_lowest_id_maximum():
    import torch
    ctx = rb.Context(0)
    try:
        g = ic_graph()
        p = rb.Pool(rb.DeviceGraph(ctx, g, "IC"))
        rng = np.random.default_rng(5)
        for n_max in [1, 3, 1000]:
            c = rng.integers(0, n_max, g.n).astype(np.uint32)
            t = torch.from_numpy(c.view(np.int32)).cuda()
            v, gain = p.shard_pick(t.data_ptr())
            assert gain == int(c.max()) and v == int(np.flatnonzero(c == c.max())[0])
        # counts above 2^31 stay unsigned
        c = np.zeros(g.n, np.uint32)
        c[77] = 3_000_000_000
        c[5] = 2_999_999_999
        v, gain = p.shard_pick(torch.from_numpy(c.view(np.int32)).cuda().data_ptr())
        assert (v, gain) == (77, 3_000_000_000)
        # misaligned arrays are refused
        t = torch.zeros(g.n + 4, dtype=torch.int32, device="cuda")
        with pytest.raises(rb.RipError):
            p.shard_pick(t.data_ptr() + 4)
        # a cover before any begin is refused
        with pytest.raises(rb.RipError):
            p.shard_cover(0, 1, t.data_ptr())
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
        seeds, rec = imm_sharded(sh, k, eps, 1.0, seed, group=dist.group.WORLD)
        assert seeds == ref_seeds and rec["theta"] == ref.theta and rec["f"] == ref.f
    finally:
        dist.destroy_process_group()
        ctx.close()
