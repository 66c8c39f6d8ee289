"""Parity of the CUDA path with the oracle and with the reference's golden
outputs.  Integer work must be bit-exact: sampled sets (vs the CPU
restatement), seed sequences, gains, coverage and theta (vs the reference's
FindMostInfluentialSet / IMM math)."""
import numpy as np
import pytest

import ripples_b200 as rb
from conftest import csr_of, karate
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SAMPLERS = [(rb.SAMPLER_PLAIN, 64), (rb.SAMPLER_FUSED, 64), (rb.SAMPLER_FUSED, 128),
            (rb.SAMPLER_FUSED, 256)]


def ic_graph(scale=12, deg=8, hi=0.3, seed=1):
    return rb.HostGraph.rmat(scale, deg << scale, seed=seed).with_weights(
        rb.WEIGHTS_UNIFORM, seed=seed + 100, lo=0.0, hi=hi)


def lt_graph(scale=12, deg=8, seed=2):
    return rb.HostGraph.rmat(scale, deg << scale, seed=seed).with_weights(
        rb.WEIGHTS_LT_NORMALIZED, seed=seed + 100)


def oracle_sets(g, model, seed, first, count):
    thr = O.pack(model, g.index, g.weights)
    return O.sample(model, g.n, g.index, g.src, thr, seed, first, count)


def device_pool(ctx, g, model, colors=64):
    dg = rb.DeviceGraph(ctx, g, model)
    p = rb.Pool(dg)
    p.configure(colors=colors)
    return dg, p


def assert_same_sets(off_a, vtx_a, off_b, vtx_b):
    assert np.array_equal(off_a, off_b)
    assert np.array_equal(vtx_a, vtx_b)


def test_thresholds_match_oracle(ctx):
    for model, g in [("IC", ic_graph(10)), ("LT", lt_graph(10))]:
        dg = rb.DeviceGraph(ctx, g, model)
        assert np.array_equal(dg.thresholds(), O.pack(model, g.index, g.weights))
        dg.close()


@pytest.mark.parametrize("sampler,colors,occupancy", [s + (0,) for s in SAMPLERS] +
                         [(rb.SAMPLER_PLAIN, 64, 5)])
def test_ic_sets_bit_exact(ctx, sampler, colors, occupancy):
    g = ic_graph()
    dg, p = device_pool(ctx, g, "IC", colors)
    p.plain_occupancy(occupancy)
    p.sample(3000, seed=7, sampler=sampler)
    off, vtx = p.export()
    ooff, ovtx, ost = oracle_sets(g, "IC", 7, 0, 3000)
    assert_same_sets(off, vtx, ooff, ovtx)
    st = p.stats()
    assert st[2] == 3000 and st[3] == len(vtx)
    assert st[4] == ost[0]  # per-set expansions = sum of set sizes
    assert st[5] == ost[1]  # per-set in-edges read
    if sampler == rb.SAMPLER_PLAIN:
        assert st[0] == st[4] and st[1] == st[5]
    else:
        assert st[0] <= st[4] and st[1] <= st[5]  # fusion never reads more


def test_karate_ic_bit_exact(ctx):
    g = karate(weight=0.5)
    for sampler, colors in SAMPLERS:
        dg, p = device_pool(ctx, g, "IC", colors)
        p.sample(2000, seed=1, sampler=sampler)
        off, vtx = p.export()
        ooff, ovtx, _ = oracle_sets(g, "IC", 1, 0, 2000)
        assert_same_sets(off, vtx, ooff, ovtx)


def test_lt_sets_bit_exact(ctx):
    g = lt_graph()
    dg, p = device_pool(ctx, g, "LT")
    p.sample(4000, seed=3)
    off, vtx = p.export()
    ooff, ovtx, ost = oracle_sets(g, "LT", 3, 0, 4000)
    assert_same_sets(off, vtx, ooff, ovtx)
    assert p.stats()[4] == ost[0]


def test_lt_long_in_lists_match_oracle(ctx):
    # in-lists past 1024 edges: several rounds of the walk's 32-ary search
    g = lt_graph(14, deg=16, seed=5)
    assert np.diff(g.index).max() > 1024
    dg = rb.DeviceGraph(ctx, g, "LT")
    p = rb.Pool(dg)
    p.sample(6000, seed=13)
    off, vtx = p.export()
    ooff, ovtx, ost = oracle_sets(g, "LT", 13, 0, 6000)
    assert_same_sets(off, vtx, ooff, ovtx)
    assert p.stats()[4] == ost[0]


def test_lt_long_walks_retry(ctx):
    """A chain 0 <- 1 <- ... <- n-1 with weight 1: walks from high roots run
    past the default per-warp queue, forcing the widen-and-retry path."""
    n = 40000
    g = rb.HostGraph.from_edges(n, np.arange(1, n), np.arange(0, n - 1),
                                np.ones(n - 1, np.float32))
    dg, p = device_pool(ctx, g, "LT")
    p.sample(64, seed=5)
    off, vtx = p.export()
    ooff, ovtx, _ = oracle_sets(g, "LT", 5, 0, 64)
    assert_same_sets(off, vtx, ooff, ovtx)
    assert np.diff(off).max() > 16384


def test_ic_giant_sets_retry(ctx):
    """p = 1 on a strongly connected graph: every set is the whole graph, far
    above the first pool-size estimate and the default queue."""
    n = 30000
    src = np.concatenate([np.arange(n), np.arange(n)])
    dst = np.concatenate([(np.arange(n) + 1) % n, (np.arange(n) + 7) % n])
    g = rb.HostGraph.from_edges(n, src, dst, np.ones(2 * n, np.float32))
    for sampler, colors in [(rb.SAMPLER_PLAIN, 64), (rb.SAMPLER_FUSED, 64)]:
        dg, p = device_pool(ctx, g, "IC", colors)
        p.sample(70, seed=2, sampler=sampler)
        off, vtx = p.export()
        assert np.all(np.diff(off) == n)
        ooff, ovtx, _ = oracle_sets(g, "IC", 2, 0, 70)
        assert_same_sets(off, vtx, ooff, ovtx)


def test_fused_log_overflow_falls_back(ctx):
    g = ic_graph(11, hi=0.5)
    dg, p = device_pool(ctx, g, "IC", 64)
    p.configure(colors=64, slots=4, log_capacity=8)
    p.sample(500, seed=9, sampler=rb.SAMPLER_FUSED)
    off, vtx = p.export()
    ooff, ovtx, _ = oracle_sets(g, "IC", 9, 0, 500)
    assert_same_sets(off, vtx, ooff, ovtx)


def test_sets_depend_only_on_set_id(ctx):
    g = ic_graph(11)
    dg, p1 = device_pool(ctx, g, "IC")
    p1.sample(1000, seed=4)
    p2 = rb.Pool(dg)
    p2.sample(300, seed=4, sampler=rb.SAMPLER_PLAIN)
    p2.sample(700, seed=4, sampler=rb.SAMPLER_FUSED)
    a = p1.export()
    b = p2.export()
    assert_same_sets(*a, *b)
    # a different seed gives different sets
    p3 = rb.Pool(dg)
    p3.sample(1000, seed=5)
    assert not np.array_equal(p3.export()[1][:1000], a[1][:1000])


def empty_graph(ctx, n):
    g = rb.HostGraph(n, np.zeros(n + 1, np.uint64), np.zeros(0, np.uint32),
                     np.zeros(0, np.float32))
    return rb.DeviceGraph(ctx, g, "IC")


def test_selection_matches_reference_golden(ctx, golden_selection):
    for i, c in enumerate(golden_selection):
        dg = empty_graph(ctx, c["n"])
        p = rb.Pool(dg)
        p.import_sets(c["off"], c["vtx"])
        f, seeds, gains = p.select(c["k"], tiebreak=rb.TIE_REF_HEAP)
        assert seeds.tolist() == c["seeds"].tolist(), f"case {i}"
        assert f == c["f"], f"case {i}"
        of, oseeds, ogains, _ = O.select(c["n"], c["off"], c["vtx"], c["k"], 0)
        assert gains.tolist() == ogains.tolist()
        p.close()
        dg.close()


def test_counting_known_answers_on_device(ctx, golden_kat):
    kat = golden_kat
    off, vtx = csr_of(kat["sets"])
    dg = empty_graph(ctx, kat["n"])
    p = rb.Pool(dg)
    p.import_sets(off, vtx)
    assert p.count().tolist() == kat["counts"]
    f, seeds, gains = p.select(2, tiebreak=rb.TIE_LOWEST_ID)
    assert seeds.tolist() == [2, 1]
    # counts after covering seed 2 (the last update before k was reached)
    assert p.select_counts().tolist() == kat["after_seed_2"]
    f, seeds, gains = p.select(3, tiebreak=rb.TIE_LOWEST_ID)
    assert seeds.tolist()[:2] == [2, 1]
    assert p.select_counts().tolist() == kat["after_seed_1"]
    # heap tie-break on the same sets agrees with the oracle (= reference)
    f, seeds, gains = p.select(3, tiebreak=rb.TIE_REF_HEAP)
    of, oseeds, ogains, _ = O.select(kat["n"], off, vtx, 3, 0)
    assert seeds.tolist() == oseeds.tolist() and gains.tolist() == ogains.tolist()


@pytest.mark.parametrize("tiebreak", [rb.TIE_REF_HEAP, rb.TIE_LOWEST_ID])
def test_selection_on_sampled_pool(ctx, tiebreak):
    g = ic_graph(12, hi=0.2)
    dg, p = device_pool(ctx, g, "IC")
    p.sample(20000, seed=11)
    off, vtx = p.export()
    for k, S in [(50, 20000), (20, 7000), (1, 20000)]:
        f, seeds, gains = p.select(k, num_sets=S, tiebreak=tiebreak)
        of, oseeds, ogains, _ = O.select(g.n, off[: S + 1], vtx[: int(off[S])], k, tiebreak)
        assert seeds.tolist() == oseeds.tolist()
        assert gains.tolist() == ogains.tolist()
        assert f == of


@pytest.mark.parametrize("guess", [1, 50, 0, 100])
def test_reference_heap_candidate_fetch(ctx, guess):
    # many vertices and heavy ties (LT walks are short, most counts are 1-3):
    # whatever threshold the first fetch of a pick uses (too low: more items
    # than the fetch holds; too high: a second, exact fetch), the seeds equal
    # the reference heap's (the oracle's)
    g = lt_graph(14, 4, seed=21)
    dg, p = device_pool(ctx, g, "LT")
    p.sample(30000, seed=5)
    p.select_guess(guess)
    off, vtx = p.export()
    for k, S in [(300, 30000), (40, 9000)]:
        f, seeds, gains = p.select(k, num_sets=S, tiebreak=rb.TIE_REF_HEAP)
        of, oseeds, ogains, _ = O.select(g.n, off[: S + 1], vtx[: int(off[S])], k, 0)
        assert seeds.tolist() == oseeds.tolist()
        assert gains.tolist() == ogains.tolist() and f == of
    # the counts after the last update step (every seed but a k-th one
    # covered) come back on demand
    covering = set(oseeds.tolist()[:-1] if len(oseeds) == k else oseeds.tolist())
    want = np.zeros(g.n, np.int64)
    for s in range(S):
        members = vtx[int(off[s]):int(off[s + 1])]
        if not covering.intersection(members.tolist()):
            np.add.at(want, members.astype(np.int64), 1)
    assert p.select_counts().tolist() == want.tolist()


@pytest.mark.parametrize("scale,hi", [(13, 0.2), (11, 0.5)])
def test_giant_component_sets_bit_exact(ctx, scale, hi):
    """Supercritical IC (R-MAT, degree 16): a large share of the sets hold a
    large share of the graph and go to the grid-wide multi-colour BFS in
    batches of up to 256; they must equal the oracle's sets."""
    g = rb.HostGraph.rmat(scale, 16 << scale, seed=3).with_weights(
        rb.WEIGHTS_UNIFORM, seed=4, lo=0.0, hi=hi)
    dg, p = device_pool(ctx, g, "IC", 64)
    p.work_caps(1 << 12, 1 << 16)
    p.sample(700, seed=21, sampler=rb.SAMPLER_PLAIN)
    p.sample(300, seed=21, sampler=rb.SAMPLER_FUSED)
    off, vtx = p.export()
    ooff, ovtx, ost = oracle_sets(g, "IC", 21, 0, 1000)
    assert_same_sets(off, vtx, ooff, ovtx)
    lens = np.diff(off.astype(np.int64))
    assert (lens > g.n // 20).sum() > 32  # the giant sets were there
    st = p.stats()
    assert st[2] == 1000 and st[3] == len(vtx) and st[5] == ost[1]


def test_selection_stops_when_all_covered(ctx):
    dg = empty_graph(ctx, 10)
    p = rb.Pool(dg)
    off, vtx = csr_of([[1, 2], [2, 3], [3], [9]])
    p.import_sets(off, vtx)
    f, seeds, gains = p.select(8)
    of, oseeds, ogains, _ = O.select(10, off, vtx, 8, 0)
    assert f == 1.0 == of and seeds.tolist() == oseeds.tolist() and gains.sum() == 4
    f, seeds, gains = p.select(0)
    assert len(seeds) == 0 and f == 0.0


@pytest.mark.parametrize("sampler", [rb.SAMPLER_PLAIN, rb.SAMPLER_FUSED])
def test_imm_ic_matches_oracle(ctx, sampler):
    # the 2^14-vertex IC configuration: R-MAT 2^14 / 2^18 draws, p ~ U(0, 0.1)
    g = rb.HostGraph.rmat(14, 1 << 18, seed=0).with_weights(rb.WEIGHTS_UNIFORM, seed=1,
                                                             lo=0.0, hi=0.1)
    gen = rb.B200RRRGenerator(g, "IC", seed=0, ctx=ctx, sampler=sampler)
    CFG = rb.IMMConfiguration(k=20, epsilon=0.5, diffusionModel="IC")
    rec = rb.IMMExecutionRecord()
    seeds = rb.IMM(g, CFG, 1.0, gen, rec)
    thr = O.pack("IC", g.index, g.weights)
    o = O.imm("IC", g.n, g.index, g.src, thr, 20, 0.5, seed=0)
    assert seeds == o["seeds"]
    assert rec.Theta == o["theta"]
    assert rec.ThetaPrimeDeltas == o["deltas"]
    assert rec.TotalSets == o["total_sets"]


def test_imm_lt_matches_oracle(ctx):
    g = lt_graph(13, 8, seed=9)
    gen = rb.B200RRRGenerator(g, "LT", seed=3, ctx=ctx)
    CFG = rb.IMMConfiguration(k=10, epsilon=0.5, diffusionModel="LT")
    rec = rb.IMMExecutionRecord()
    seeds = rb.IMM(g, CFG, 1.0, gen, rec)
    thr = O.pack("LT", g.index, g.weights)
    o = O.imm("LT", g.n, g.index, g.src, thr, 10, 0.5, seed=3)
    assert seeds == o["seeds"] and rec.Theta == o["theta"]
    assert rec.ThetaPrimeDeltas == o["deltas"]


def test_find_most_influential_set_host_lists(ctx, golden_selection):
    c = golden_selection[-1]
    sets = [c["vtx"][c["off"][i]:c["off"][i + 1]] for i in range(len(c["off"]) - 1)]
    G = rb.HostGraph(c["n"], np.zeros(c["n"] + 1, np.uint64), np.zeros(0, np.uint32),
                     np.zeros(0, np.float32))
    CFG = rb.IMMConfiguration(k=c["k"])
    f, seeds = rb.FindMostInfluentialSet(G, CFG, sets, ctx=ctx)
    assert seeds == c["seeds"].tolist() and f == c["f"]


def test_errors_are_reported(ctx):
    g = ic_graph(8)
    dg, p = device_pool(ctx, g, "IC")
    p.sample(10)
    with pytest.raises(rb.RipError):
        p.select(5, num_sets=11)
    with pytest.raises(rb.RipError):
        p.configure(colors=96)
    bad = rb.HostGraph(g.n, g.index, g.src.copy(), g.weights)
    bad.src[0] = g.n + 5
    with pytest.raises(rb.RipError):
        rb.DeviceGraph(ctx, bad, "IC")
    dg2 = empty_graph(ctx, 4)
    p2 = rb.Pool(dg2)
    off, vtx = csr_of([[1, 7]])
    with pytest.raises(rb.RipError):
        p2.import_sets(off, vtx)


@pytest.mark.parametrize("model,weights,lo,hi", [("IC", rb.WEIGHTS_UNIFORM, 0.0, 0.1),
                                                 ("IC", rb.WEIGHTS_WC, 0.0, 1.0),
                                                 ("LT", rb.WEIGHTS_LT_NORMALIZED, 0.0, 1.0)])
def test_device_graph_construction_matches_host(ctx, model, weights, lo, hi):
    scale, draws = 12, 16 << 12
    hg = rb.HostGraph.rmat(scale, draws, seed=3).with_weights(weights, seed=4, lo=lo, hi=hi)
    dg = rb.DeviceGraph.rmat_on_device(ctx, scale, draws, model, weights, seed=3,
                                       weight_seed=4, lo=lo, hi=hi)
    idx, src = dg.export()
    assert np.array_equal(idx, hg.index) and np.array_equal(src, hg.src)
    assert np.array_equal(dg.thresholds(), O.pack(model, hg.index, hg.weights))
    dg.close()
    eg = rb.HostGraph.erdos_renyi(3000, 40000, seed=6).with_weights(weights, seed=4, lo=lo, hi=hi)
    de = rb.DeviceGraph.erdos_renyi_on_device(ctx, 3000, 40000, model, weights, seed=6,
                                              weight_seed=4, lo=lo, hi=hi)
    idx, src = de.export()
    assert np.array_equal(idx, eg.index) and np.array_equal(src, eg.src)
    assert np.array_equal(de.thresholds(), O.pack(model, eg.index, eg.weights))
    de.close()


@pytest.mark.parametrize("weights", [rb.WEIGHTS_UNIFORM, rb.WEIGHTS_WC])
@pytest.mark.parametrize("sampler", [rb.SAMPLER_PLAIN, rb.SAMPLER_FUSED])
@pytest.mark.parametrize("heavy_batch", [0, 1])
def test_big_set_path_bit_exact(ctx, weights, sampler, heavy_batch):
    """Tiny edge-work budgets send most sets to the heavy-set samplers (one
    CTA per set, or the grid-wide multi-colour BFS); the sets must not
    change."""
    g = rb.HostGraph.rmat(12, 16 << 12, seed=8).with_weights(weights, seed=9, lo=0.0, hi=0.4)
    dg, p = device_pool(ctx, g, "IC", 64)
    p.work_caps(64, 256)
    p.heavy_batch(heavy_batch)
    p.sample(3000, seed=12, sampler=sampler)
    off, vtx = p.export()
    ooff, ovtx, ost = oracle_sets(g, "IC", 12, 0, 3000)
    assert_same_sets(off, vtx, ooff, ovtx)
    st = p.stats()
    assert st[2] == 3000 and st[4] == ost[0] and st[5] == ost[1]


@pytest.mark.parametrize("n,max_count,seed", [(1, 3, 0), (2, 1, 1), (37, 2, 2), (5000, 3, 3),
                                              (1 << 20, 5, 4), ((1 << 20) + 12345, 1000, 5)])
def test_device_heap_is_libstdcxx_make_heap(ctx, n, max_count, seed):
    """rip_select builds its max-heap on the device; it must equal
    std::make_heap element for element (ties included)."""
    assert rb._lib.lib.rip_selftest_heap_device(ctx.h, n, max_count, seed) == 1


@pytest.mark.parametrize("model", ["IC", "LT"])
@pytest.mark.parametrize("case", ["no_edges", "pair", "triangle", "isolated_tail"])
def test_corner_graphs_match_oracle(ctx, model, case):
    """Graphs at the edges of the input space: no edges at all (every set is
    its root), two and three vertices, and a small graph whose last vertices
    have no in- or out-edges.  Sets, IMM seeds and theta equal the oracle's,
    under every sampler and both tie-breaks."""
    if case == "no_edges":
        g = rb.HostGraph.from_edges(5, [], [], np.zeros(0, np.float32))
    elif case == "pair":
        g = rb.HostGraph.from_edges(2, [0, 1], [1, 0], np.array([0.9, 0.4], np.float32))
    elif case == "triangle":
        g = rb.HostGraph.from_edges(3, [0, 1, 2, 0], [1, 2, 0, 2],
                                    np.array([0.7, 0.5, 1.0, 0.3], np.float32))
    else:
        e = rb.HostGraph.rmat(6, 256, seed=4)
        src, dst = e.transpose_edges()
        g = rb.HostGraph.from_edges(80, src, dst, np.full(len(src), 0.3, np.float32))
    if model == "LT":
        g = g.with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=5) if g.m else g
    thr = O.pack(model, g.index, g.weights)
    samplers = [rb.SAMPLER_PLAIN, rb.SAMPLER_FUSED] if model == "IC" else [rb.SAMPLER_AUTO]
    for sampler in samplers:
        dg, p = device_pool(ctx, g, model)
        p.sample(700, seed=2, sampler=sampler)
        off, vtx = p.export()
        ooff, ovtx, _ = O.sample(model, g.n, g.index, g.src, thr, 2, 0, 700)
        assert_same_sets(off, vtx, ooff, ovtx)
        for tie in (rb.TIE_REF_HEAP, rb.TIE_LOWEST_ID):
            k = min(3, g.n)
            f, seeds, gains = p.select(k + 2, tiebreak=tie)  # k beyond what can add coverage
            of, oseeds, ogains, _ = O.select(g.n, off, vtx, k + 2, tie)
            assert seeds.tolist() == oseeds.tolist() and f == of
        p.close()
        dg.close()
    for tie in (rb.TIE_REF_HEAP, rb.TIE_LOWEST_ID):
        dg = rb.DeviceGraph(ctx, g, model)
        q = rb.Pool(dg)
        seeds, rec = q.imm(2, 0.5, seed=3, tiebreak=tie)
        o = O.imm(model, g.n, g.index, g.src, thr, 2, 0.5, seed=3, tiebreak=tie)
        assert seeds.tolist() == o["seeds"] and rec.theta == o["theta"], (case, tie)
        q.close()
        dg.close()


def mixed_uniform_graph(scale=12, deg=16, seed=31):
    """Weighted cascade on two vertices in three, U(0, 0.3) per edge on the
    rest: uniform in-lists hold about two thirds of the edges, so the graph
    keeps per-vertex uniform thresholds and the samplers meet both kinds of
    list in one set."""
    g = rb.HostGraph.rmat(scale, deg << scale, seed=seed)
    wc = g.with_weights(rb.WEIGHTS_WC).weights
    un = g.with_weights(rb.WEIGHTS_UNIFORM, seed=seed + 1, lo=0.0, hi=0.3).weights
    dst = np.repeat(np.arange(g.n), np.diff(g.index).astype(np.int64))
    return rb.HostGraph(g.n, g.index, g.src, np.where(dst % 3 == 0, un, wc).astype(np.float32))


@pytest.mark.parametrize("path", ["plain", "cta_per_set", "multi"])
def test_uniform_thresholds_match_oracle(ctx, path):
    g = mixed_uniform_graph()
    dg = rb.DeviceGraph(ctx, g, "IC")
    assert dg.uniform_thresholds()  # built at upload, on
    ooff, ovtx, ost = oracle_sets(g, "IC", 17, 0, 3000)
    try:
        for enable in (True, False):
            dg.uniform_thresholds(enable)
            p = rb.Pool(dg)
            if path == "cta_per_set":
                p.work_caps(64, 1 << 23)  # nearly every set goes to the CTA-per-set kernel
                p.heavy_batch(0)
            if path == "multi":
                rb.sample_multi(ctx, [p], [17], [3000])
            else:
                p.sample(3000, seed=17, sampler=rb.SAMPLER_PLAIN)
            off, vtx = p.export()
            assert_same_sets(off, vtx, ooff, ovtx)
            st = p.stats()
            assert st[5] == ost[1]  # coins drawn for every in-edge of every member
            # records of uniform lists are skipped only when switched on
            assert (st[6] > 0) == enable and (st[7] > 0) == enable
            p.close()
    finally:
        dg.close()


def test_uniform_thresholds_only_where_they_pay(ctx):
    # U(0, 0.3) per edge: only in-lists of one edge are uniform, far from half
    # of the edges, so no per-vertex array is kept
    dg = rb.DeviceGraph(ctx, ic_graph(12), "IC")
    assert not dg.uniform_thresholds()
    dg.close()
    # weighted cascade: every list is uniform, and a reverse BFS is at most
    # critical (an edge's source has one live in-edge on average, or none)
    g = rb.HostGraph.rmat(12, 8 << 12, seed=3).with_weights(rb.WEIGHTS_WC)
    dg = rb.DeviceGraph(ctx, g, "IC")
    assert dg.uniform_thresholds()
    lam = np.bincount(np.repeat(np.arange(g.n), np.diff(g.index).astype(np.int64)),
                      weights=g.weights.astype(np.float64), minlength=g.n)
    assert abs(dg.branching - lam[g.src].mean()) < 1e-3 and dg.branching <= 1.0 + 1e-6
    dg.close()
    # LT graphs never keep one
    dg = rb.DeviceGraph(ctx, lt_graph(10), "LT")
    assert not dg.uniform_thresholds()
    dg.close()


@pytest.mark.parametrize("threads", [128, 256, 512, 1024])
def test_cta_per_set_block_shapes_match_oracle(ctx, threads):
    # R-MAT 2^16 with 32 draws per vertex: the largest in-list passes 1024
    # 8-edge coin blocks, so every block shape sweeps a list with the whole
    # CTA
    g = mixed_uniform_graph(scale=16, deg=32, seed=41)
    assert np.diff(g.index).max() >= 8 * 1024
    dg = rb.DeviceGraph(ctx, g, "IC")
    p = rb.Pool(dg)
    try:
        p.work_caps(64, 1 << 23)  # nearly every set goes to the CTA-per-set kernel
        p.heavy_batch(0)
        p.heavy_block(threads)
        p.sample(600, seed=23, sampler=rb.SAMPLER_PLAIN)
        off, vtx = p.export()
        ooff, ovtx, _ = oracle_sets(g, "IC", 23, 0, 600)
        assert_same_sets(off, vtx, ooff, ovtx)
    finally:
        p.close()
        dg.close()
