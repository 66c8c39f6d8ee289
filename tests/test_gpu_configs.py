"""Parity on the benchmarked configurations themselves, on the device.

* LT, R-MAT 2^20 (16 * 2^20 draws, in-weights U(0,1) normalised per
  destination), k = 50, epsilon = 0.3: the device IMM (rip_imm_pool) returns
  the oracle's seeds, theta, round deltas and f, under both tie-breaks.
* The same configuration's spread: the device IMM's seeds against the seeds of
  the reference's own sequential IMM (include/ripples/imm.h:671-752, built from
  its sources), both measured by one Monte Carlo simulator with common random
  numbers.  The reference's LT simulator (diffusion_simulation.h:129-178)
  transposes the whole graph on every replica (:135), so at 2^20 vertices it
  runs minutes per replica; the device LT simulator stands in for it here.  It
  equals the oracle replica for replica, and the oracle agrees with the
  reference simulator on smaller graphs (tests/test_gpu_spread.py,
  tests/test_oracle.py).
* IC, R-MAT 2^24 (32 * 2^24 draws), weighted cascade p = 1/in-degree: 4096
  set ids spread over the first 1.5 M sets (the size of one IMM's pool at
  k = 100, epsilon = 0.13), device sets bit-exact against the oracle's.
* The device sampler against the reference's own sampler in distribution on
  R-MAT 2^16 with weighted cascade (2 M sets a side).
"""
import ctypes
import os

import numpy as np
import pytest

import ripples_b200 as rb
from conftest import assert_same_distribution
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LT20 = dict(scale=20, draws=16 << 20, k=50, eps=0.3)


@pytest.fixture(scope="module")
def lt20():
    g = rb.HostGraph.rmat(LT20["scale"], LT20["draws"], 0.57, 0.19, 0.19, seed=0)
    return g.with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=1)


@pytest.fixture(scope="module")
def lt20_device(ctx, lt20):
    dg = rb.DeviceGraph(ctx, lt20, "LT")
    yield dg
    dg.close()


@pytest.mark.parametrize("tiebreak", [rb.TIE_REF_HEAP, rb.TIE_LOWEST_ID])
def test_lt20_imm_matches_oracle(lt20, lt20_device, tiebreak):
    thr = O.pack("LT", lt20.index, lt20.weights)
    pool = rb.Pool(lt20_device)
    try:
        for seed in (1000004, 7):
            pool.clear()
            seeds, rec = pool.imm(LT20["k"], LT20["eps"], 1.0, seed=seed, tiebreak=tiebreak)
            o = O.imm("LT", lt20.n, lt20.index, lt20.src, thr, LT20["k"], LT20["eps"], seed=seed,
                      tiebreak=0 if tiebreak == rb.TIE_REF_HEAP else 1)
            assert seeds.tolist() == o["seeds"]
            assert rec.theta == o["theta"] and rec.total_sets == o["total_sets"]
            assert [rec.theta_prime_deltas[i] for i in range(rec.num_rounds)] == o["deltas"]
            assert rec.f == o["f"]
    finally:
        pool.close()


def test_lt20_spread_within_one_percent_of_reference(ctx, lt20, lt20_device, tmp_path):
    R = O.reference()
    if R is None:
        pytest.skip("oracle/_ref not built")
    path = str(tmp_path / "lt20.bin")
    lt20.write_binary(path, backward=True)
    rg = R.ref_graph_load(path.encode())
    runs = 4
    try:
        ref_sets = []
        for s in range(runs):
            out = np.zeros(LT20["k"], np.uint32)
            ns = R.ref_imm_sequential(rg, 1, LT20["k"], LT20["eps"], s, out.ctypes.data)
            assert ns == LT20["k"]
            ref_sets.append(out.copy())
    finally:
        R.ref_graph_free(rg)
    pool = rb.Pool(lt20_device)
    ours = []
    try:
        for s in range(runs):
            pool.clear()
            seeds, _ = pool.imm(LT20["k"], LT20["eps"], 1.0, seed=1000004 + s)
            ours.append(seeds.copy())
    finally:
        pool.close()
    fwd = rb.DeviceGraph(ctx, lt20.forward(), "IC")
    try:
        # common random numbers: every seed set sees the same replicas
        reps = 4000
        spread = lambda sd: rb.spread_lt(fwd, lt20_device, sd, reps, seed=11)
        s_ref = [spread(sd) for sd in ref_sets]
        s_our = [spread(sd) for sd in ours]
    finally:
        fwd.close()
    mean_ref, mean_our = float(np.mean(s_ref)), float(np.mean(s_our))
    print("reference seeds' spread", s_ref, "device seeds' spread", s_our)
    assert abs(mean_our - mean_ref) / mean_ref < 0.01, (s_our, s_ref)


def test_ic24_wc_strided_sets_match_oracle(ctx):
    scale, draws, seed = 24, 32 << 24, 1000004
    n, idx, src, w = O.rmat_graph(scale, draws, seed=0, weights="wc")
    thr = O.pack("IC", idx, w)
    dg = rb.DeviceGraph.rmat_on_device(ctx, scale, draws, "IC", rb.WEIGHTS_WC, seed=0)
    pool = rb.Pool(dg)
    try:
        assert dg.n == n and dg.m == len(src)
        total = 1_500_000
        pool.sample(total, seed=seed)
        ids = np.linspace(0, total - 1, 4096).astype(np.uint64)
        off, vtx = pool.export()
        ooff, ovtx = O.sample_ids("IC", n, idx, src, thr, seed, ids)
        for j, i in enumerate(ids.tolist()):
            got = np.sort(vtx[off[i]:off[i + 1]])
            assert np.array_equal(got, ovtx[ooff[j]:ooff[j + 1]]), i
    finally:
        pool.close()
        dg.close()


def test_wc16_device_sampler_matches_reference_distribution(ctx, golden_wc16):
    z = golden_wc16
    g = rb.HostGraph(z["n"], z["index"], z["src"], z["w"])
    dg = rb.DeviceGraph(ctx, g, "IC")
    pool = rb.Pool(dg)
    try:
        nsets = int(z["nsets"][0])
        pool.sample(nsets, seed=2024)
        off, vtx = pool.export()
        assert_same_distribution(np.bincount(vtx, minlength=z["n"]), np.diff(off),
                                 z["freq"], z["size_hist"])
    finally:
        pool.close()
        dg.close()
