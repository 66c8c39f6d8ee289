"""OPIM-C on the device: rip_coverage against the oracle's FindCoverage, and
rip_opimc_pool against the oracle's OPIM-C (same pools, so the same seeds,
final theta and rounds); the oracle's OPIM-C is pinned to the reference's
opimc tool in tests/test_spread.py."""
import numpy as np
import pytest

import ripples_b200 as rb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def ic_graph(scale, deg, hi, seed):
    return rb.HostGraph.rmat(scale, deg << scale, seed=seed).with_weights(
        rb.WEIGHTS_UNIFORM, seed=seed + 100, lo=0.0, hi=hi)


def test_coverage_matches_oracle(ctx):
    g = ic_graph(12, 8, 0.3, 3)
    dg = rb.DeviceGraph(ctx, g, "IC")
    p = rb.Pool(dg)
    try:
        p.sample(3000, seed=5)
        off, vtx = p.export()
        rng = np.random.default_rng(1)
        for k in [0, 1, 3, 20, 200]:
            seeds = rng.integers(0, g.n, size=k).astype(np.uint32)
            for S in [0, 1, 777, 3000]:
                assert p.coverage(seeds, S) == O.find_coverage(off[: S + 1], vtx, seeds)
        with pytest.raises(rb.RipError):
            p.coverage([0], 3001)       # more sets than the pool holds
        with pytest.raises(rb.RipError):
            p.coverage([g.n], 10)       # seed out of range
    finally:
        p.close()
        dg.close()


@pytest.mark.parametrize("model,eps,tiebreak", [("IC", 0.5, rb.TIE_REF_HEAP),
                                                ("IC", 0.2, rb.TIE_REF_HEAP),
                                                ("IC", 0.2, rb.TIE_LOWEST_ID),
                                                ("LT", 0.2, rb.TIE_REF_HEAP)])
def test_opimc_matches_oracle(ctx, model, eps, tiebreak):
    if model == "IC":
        g = ic_graph(13, 16, 0.1, 0)
    else:
        g = rb.HostGraph.rmat(13, 16 << 13, seed=2).with_weights(rb.WEIGHTS_LT_NORMALIZED,
                                                                 seed=3)
    dg = rb.DeviceGraph(ctx, g, model)
    r1, r2 = rb.Pool(dg), rb.Pool(dg)
    try:
        seeds, rec = rb.opimc(r1, r2, 20, eps, 0.05, seed=7, tiebreak=tiebreak)
        thr = O.pack(model, g.index, g.weights)
        ref = O.opimc(model, g.n, g.index, g.src, thr, 20, eps, 0.05, seed=7,
                      tiebreak=0 if tiebreak == rb.TIE_REF_HEAP else 1)
        assert seeds.tolist() == ref["seeds"]
        assert rec.theta == ref["theta"] and rec.rounds == ref["rounds"]
        assert rec.theta_zero == ref["theta_zero"] and rec.theta_max == ref["theta_max"]
        assert r1.num_sets == r2.num_sets == rec.theta
    finally:
        r1.close()
        r2.close()
        dg.close()
