"""The device forward spread simulators (rip_spread_ic, rip_spread_lt):
every replica's reached count bit-exact against the oracle's restatement,
and the mean against the spread the reference's own simulator measured
(golden)."""
import json
import os
import sys

import numpy as np
import pytest

import ripples_b200 as rb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def forward_device(ctx, g):
    return rb.DeviceGraph(ctx, g.forward(), "IC")


def oracle_spread(g, seeds, replicas, seed):
    f = g.forward()
    thr = O.pack("IC", f.index, f.weights)
    return O.spread_ic(f.n, f.index, f.src, thr, seeds, replicas, seed=seed)


@pytest.mark.parametrize("scale,deg,hi,seeds,replicas", [
    (10, 8, 0.3, [0, 1, 2, 3], 256),            # subcritical
    (12, 16, 0.1, [0, 16, 256, 8, 32, 7], 128),  # supercritical: giant cascades
    (12, 8, None, [3], 16),                     # p = 1 on every edge: the seed's closure
    (11, 8, 0.2, [9, 9, 4, 9], 64),             # a repeated seed counts once
])
def test_spread_bit_exact_vs_oracle(ctx, scale, deg, hi, seeds, replicas):
    g = rb.HostGraph.rmat(scale, deg << scale, seed=scale)
    if hi is None:
        g = rb.HostGraph(g.n, g.index, g.src, np.ones(g.m, np.float32))
    else:
        g = g.with_weights(rb.WEIGHTS_UNIFORM, seed=scale + 50, lo=0.0, hi=hi)
    dg = forward_device(ctx, g)
    try:
        mean, sizes, levels = rb.spread_ic(dg, seeds, replicas, seed=21, with_sizes=True,
                                           with_levels=True)
        f = g.forward()
        thr = O.pack("IC", f.index, f.weights)
        o_mean, o_sizes, o_levels = O.spread_ic(f.n, f.index, f.src, thr, seeds, replicas,
                                                seed=21, with_levels=True)
        assert np.array_equal(sizes, o_sizes) and np.array_equal(levels, o_levels)
        assert mean == pytest.approx(o_mean, rel=0, abs=1e-9)
        assert rb.spread_ic(dg, seeds, replicas, seed=21) == mean  # without the sizes
    finally:
        dg.close()


def test_spread_karate_bit_exact(ctx):
    from conftest import karate
    g = karate()
    dg = forward_device(ctx, g)
    try:
        _, sizes = rb.spread_ic(dg, [0, 33], 5000, seed=3, with_sizes=True)
        _, o_sizes = oracle_spread(g, [0, 33], 5000, seed=3)
        assert np.array_equal(sizes, o_sizes)
    finally:
        dg.close()


@pytest.mark.parametrize("name", ["karate_ic", "rmat12_ic", "rmat14_ic", "karate_lt",
                                  "rmat10_lt", "rmat12_lt"])
def test_spread_matches_reference_simulator(ctx, name):
    # The device mean over many replicas against the reference simulator's
    # mean for the same seeds: within 4 standard errors and within 1%.
    sys.path.insert(0, GOLDEN)
    import make_golden as M
    with open(os.path.join(GOLDEN, "spread_reference.json")) as fh:
        case = next(r for r in json.load(fh) if r["name"] == name)
    g = M.spread_graph(case)
    seeds = np.asarray(case["seeds_list"], np.uint32)
    dg = forward_device(ctx, g)
    bg = rb.DeviceGraph(ctx, g, "LT") if case["model"] == "LT" else None
    try:
        reps = 200000
        if bg is None:
            mean, sizes = rb.spread_ic(dg, seeds, reps, seed=17, with_sizes=True)
        else:
            mean, sizes = rb.spread_lt(dg, bg, seeds, reps, seed=17, with_sizes=True)
    finally:
        if bg is not None:
            bg.close()
        dg.close()
    sd = float(np.std(sizes.astype(np.float64)))
    se = sd * np.sqrt(1.0 / reps + 1.0 / case["replicas"])
    assert abs(mean - case["spread"]) <= 4 * se + 1e-9, (mean, case["spread"], se)
    assert abs(mean - case["spread"]) / case["spread"] < 0.01


@pytest.mark.parametrize("scale,deg,kind,seeds,replicas", [
    (10, 8, "normalized", [0, 8, 64, 128], 256),
    (12, 16, "normalized", [0, 1, 2, 3, 4, 5, 6, 7], 64),
    (11, 8, "partial", [3, 3, 9], 128),   # in-weights sum below 1: some keep no edge
])
def test_spread_lt_bit_exact_vs_oracle(ctx, scale, deg, kind, seeds, replicas):
    g = rb.HostGraph.rmat(scale, deg << scale, seed=scale + 1)
    if kind == "normalized":
        g = g.with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=scale + 60)
    else:
        g = g.with_weights(rb.WEIGHTS_UNIFORM, seed=scale + 60, lo=0.0, hi=0.1)
    fg, bg = forward_device(ctx, g), rb.DeviceGraph(ctx, g, "LT")
    try:
        mean, sizes, levels = rb.spread_lt(fg, bg, seeds, replicas, seed=23, with_sizes=True,
                                           with_levels=True)
        o_mean, o_sizes, o_levels = O.spread_lt(g, seeds, replicas, seed=23, with_levels=True)
        assert np.array_equal(sizes, o_sizes) and np.array_equal(levels, o_levels)
        assert mean == pytest.approx(o_mean, rel=0, abs=1e-9)
    finally:
        bg.close()
        fg.close()


def test_spread_lt_karate_bit_exact(ctx):
    from conftest import karate
    g = karate().with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=9)
    fg, bg = forward_device(ctx, g), rb.DeviceGraph(ctx, g, "LT")
    try:
        _, sizes = rb.spread_lt(fg, bg, [0, 33], 5000, seed=4, with_sizes=True)
        _, o_sizes = O.spread_lt(g, [0, 33], 5000, seed=4)
        assert np.array_equal(sizes, o_sizes)
    finally:
        bg.close()
        fg.close()


def test_spread_arguments(ctx):
    g = rb.HostGraph.rmat(8, 4 << 8, seed=1).with_weights(rb.WEIGHTS_UNIFORM, seed=2,
                                                           lo=0.0, hi=0.2)
    dg = forward_device(ctx, g)
    lt = rb.DeviceGraph(ctx, rb.HostGraph.rmat(8, 4 << 8, seed=1).with_weights(
        rb.WEIGHTS_LT_NORMALIZED, seed=2), "LT")
    try:
        assert rb.spread_ic(dg, [], 100) == 0.0
        assert rb.spread_ic(dg, [1, 2], 0) == 0.0
        with pytest.raises(rb.RipError):
            rb.spread_ic(dg, [g.n], 10)  # out of range: rejected on the host
        with pytest.raises(rb.RipError):
            rb.spread_ic(lt, [1], 10)    # IC only
        with pytest.raises(rb.RipError):
            rb.spread_lt(dg, dg, [1], 10)  # the backward graph must be the LT upload
        small = rb.DeviceGraph(ctx, rb.HostGraph.rmat(6, 4 << 6, seed=1).with_weights(
            rb.WEIGHTS_LT_NORMALIZED, seed=2), "LT")
        try:
            with pytest.raises(rb.RipError):
                rb.spread_lt(dg, small, [1], 10)  # forward and backward differ
        finally:
            small.close()
        assert rb.spread_lt(dg, lt, [1], 10) >= 1.0  # the same graph: fine
        # the context stays usable after the rejections
        assert rb.spread_ic(dg, [1], 10) >= 1.0
    finally:
        lt.close()
        dg.close()
