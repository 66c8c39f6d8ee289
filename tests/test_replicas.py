"""The N > 1 path of the benchmark: one process per GPU, each running its own
IMM queries (replicas; the path has no data-path collective), with the
whole-job figure reduced over the ranks.  Run here as two gloo ranks on CPU."""
import os
import socket
import sys
from datetime import timedelta

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        # each replica: its own sets and its own device time
        sets, ms = 1000 * (rank + 1), 10.0 * (rank + 1)
        value, t_max = bench.aggregate(sets, ms, world)
        seeds = [bench.replica_seed(rank, s) for s in range(3)]
        bench.barrier(world)
        out.put((rank, value, t_max, seeds))
    finally:
        dist.destroy_process_group()


def test_replicas_reduce_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_replica, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    # whole-job sets over the slowest rank's time, the same on every rank
    for _, value, t_max, _ in res:
        assert t_max == 20.0
        assert value == pytest.approx((1000 + 2000) / 0.020)
    # replicas sample different sets
    assert not set(res[0][3]) & set(res[1][3])


def test_reference_arm_runs_on_rank_zero_only():
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        warmup, steps = 1, 1
    # a rank other than 0 returns at once, without building or timing anything
    assert bench.reference_arm(Args(), bench.WORKLOADS["lt20"], world=2, rank=1) == 0


@pytest.mark.parametrize("workload", ["b1", "s1", "ic24_samplers", "ic24u_samplers",
                                      "ic24_sharded"])
def test_reference_arm_of_other_workloads(workload, capsys):
    # batching, serving and the comparison of this library's samplers have no
    # runnable reference counterpart: one unavailable line, exit 0, no GPU
    # path taken
    sys.path.insert(0, ROOT)
    import json
    import bench

    class Args:
        warmup, steps = 1, 1
    assert bench.reference_arm_other(Args(), bench.WORKLOADS[workload], world=1, rank=0) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unavailable"]
    assert bench.reference_arm_other(Args(), bench.WORKLOADS[workload], world=2, rank=1) == 0
