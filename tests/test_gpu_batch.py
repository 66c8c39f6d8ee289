"""Batching and serving: many pools extended in one launch, IMM queries run as
a continuous batch over shared resident pools.  Every answer must equal the
one the query gets alone (a fresh rip_imm), and the oracle's."""
import numpy as np
import pytest

import ripples_b200 as rb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def ic_graph(scale, deg=8, hi=0.1, seed=1):
    return rb.HostGraph.rmat(scale, deg << scale, seed=seed).with_weights(
        rb.WEIGHTS_UNIFORM, seed=seed + 100, lo=0.0, hi=hi)


def lt_graph(scale, deg=8, seed=2):
    return rb.HostGraph.rmat(scale, deg << scale, seed=seed).with_weights(
        rb.WEIGHTS_LT_NORMALIZED, seed=seed + 100)


def er_graph(n, m, seed=5, hi=0.05):
    return rb.HostGraph.erdos_renyi(n, m, seed=seed).with_weights(
        rb.WEIGHTS_UNIFORM, seed=seed + 100, lo=0.0, hi=hi)


@pytest.fixture(scope="module")
def graphs(ctx):
    hs = {"ic12": (ic_graph(12), "IC"), "lt12": (lt_graph(12), "LT"),
          "ic10": (ic_graph(10, hi=0.3, seed=4), "IC"), "lt13": (lt_graph(13, seed=6), "LT"),
          "er11": (er_graph(1 << 11, 1 << 14), "IC")}
    dev = {k: rb.DeviceGraph(ctx, g, m) for k, (g, m) in hs.items()}
    yield hs, dev
    for d in dev.values():
        d.close()


def test_sample_multi_equals_single_pools(ctx, graphs):
    hs, dev = graphs
    names = list(dev)
    counts = [1500, 2200, 700, 3100, 900]
    seeds = [11, 12, 13, 14, 15]
    multi = [rb.Pool(dev[k]) for k in names]
    # a first extension, then a second on top of it (set ids continue)
    rb.sample_multi(ctx, multi, seeds, counts)
    rb.sample_multi(ctx, multi, seeds, [c // 3 for c in counts])
    for k, p, s, c in zip(names, multi, seeds, counts):
        single = rb.Pool(dev[k])
        single.sample(c + c // 3, seed=s, sampler=rb.SAMPLER_PLAIN)
        a, b = p.export(), single.export()
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), k
        g, model = hs[k]
        thr = O.pack(model, g.index, g.weights)
        ooff, ovtx, _ = O.sample(model, g.n, g.index, g.src, thr, s, 0, 400)
        assert np.array_equal(a[0][:401], ooff) and np.array_equal(a[1][: len(ovtx)], ovtx)
        single.close()
    for p in multi:
        p.close()


def test_sample_multi_retries_and_heavy_sets(ctx, graphs):
    hs, dev = graphs
    # a tiny edge-work cap sends IC sets to the CTA-per-set path, and a fresh
    # pool below the pilot size starts at its minimum capacity
    pools = [rb.Pool(dev["ic10"]), rb.Pool(dev["lt12"])]
    pools[0].work_caps(64, 1 << 23)
    rb.sample_multi(ctx, pools, [3, 4], [4000, 4000])
    for p, (k, s) in zip(pools, [("ic10", 3), ("lt12", 4)]):
        g, model = hs[k]
        thr = O.pack(model, g.index, g.weights)
        ooff, ovtx, _ = O.sample(model, g.n, g.index, g.src, thr, s, 0, 4000)
        off, vtx = p.export()
        assert np.array_equal(off, ooff) and np.array_equal(vtx, ovtx), k
        p.close()


def alone(dev, name, k, eps, seed, tie):
    p = rb.Pool(dev[name])
    seeds, rec = p.imm(k, eps, seed=seed, tiebreak=tie, sampler=rb.SAMPLER_PLAIN)
    p.close()
    return seeds, rec


QUERIES = [("ic12", 20, 0.5, 0), ("lt12", 15, 0.4, 1), ("ic10", 8, 0.3, 2),
           ("lt13", 30, 0.5, 3), ("er11", 12, 0.5, 4), ("ic12", 5, 0.3, 0),
           ("lt12", 40, 0.5, 1)]


@pytest.mark.parametrize("tie", [rb.TIE_LOWEST_ID, rb.TIE_REF_HEAP])
def test_imm_batch_equals_alone(ctx, graphs, tie):
    hs, dev = graphs
    qs = [rb.Query(dev[n], k, e, seed=s, tiebreak=tie) for n, k, e, s in QUERIES]
    rb.imm_batch(ctx, qs)
    for (n, k, e, s), q in zip(QUERIES, qs):
        assert q.done and q.status == 0
        ref_seeds, ref_rec = alone(dev, n, k, e, s, tie)
        assert q.seeds.tolist() == ref_seeds.tolist(), (n, k, e)
        r = q.record
        assert r.theta == ref_rec.theta and r.num_rounds == ref_rec.num_rounds
        nr = min(r.num_rounds, 64)
        assert list(r.theta_prime_deltas[:nr]) == list(ref_rec.theta_prime_deltas[:nr])
        assert r.total_sets == ref_rec.total_sets
        assert r.f == pytest.approx(ref_rec.f, abs=0.0)


def test_imm_batch_matches_oracle(ctx, graphs):
    hs, dev = graphs
    for n, k, e, s in QUERIES[:4]:
        q = rb.Query(dev[n], k, e, seed=s, tiebreak=rb.TIE_LOWEST_ID)
        rb.imm_batch(ctx, [q])
        g, model = hs[n]
        thr = O.pack(model, g.index, g.weights)
        o = O.imm(model, g.n, g.index, g.src, thr, k, e, seed=s, tiebreak=1)
        assert q.seeds.tolist() == o["seeds"], n
        assert q.record.theta == o["theta"]


def test_server_staggered_arrivals_share_pools(ctx, graphs):
    hs, dev = graphs
    srv = rb.Server(ctx, max_active=3)
    first = [srv.submit(rb.Query(dev[n], k, e, seed=s)) for n, k, e, s in QUERIES[:4]]
    srv.tick()
    srv.tick()
    later = [srv.submit(rb.Query(dev[n], k, e, seed=s)) for n, k, e, s in QUERIES[4:]]
    active, queued = srv.pending()
    assert active <= 3
    srv.drain()
    st = srv.stats()
    # one pool per distinct (graph, seed)
    assert st["pools"] == len({(n, s) for n, _, _, s in QUERIES})
    assert st["completed"] == len(QUERIES)
    assert st["graph_launches"] > 0
    for (n, k, e, s), q in zip(QUERIES, first + later):
        assert q.done and q.status == 0
        ref_seeds, ref_rec = alone(dev, n, k, e, s, rb.TIE_LOWEST_ID)
        assert q.seeds.tolist() == ref_seeds.tolist(), (n, k, e)
        assert q.record.theta == ref_rec.theta
        assert q.latency_ms >= q.q.queue_ms >= 0
    srv.close()


def test_server_rejects_bad_query(ctx, graphs):
    hs, dev = graphs
    srv = rb.Server(ctx, max_active=2)
    bad = rb.Query(dev["ic12"], 5, 0.5)
    bad.q.epsilon = 0.0
    good = rb.Query(dev["ic12"], 5, 0.5)
    srv.submit(bad)
    srv.submit(good)
    srv.drain()
    assert bad.done and bad.status == -1
    assert good.done and good.status == 0 and len(good.seeds) == 5
    srv.close()


def test_autotune_picks_a_configuration_and_sets_stay_exact(ctx):
    # a supercritical IC graph (heavy sets) and an LT graph
    g = rb.HostGraph.rmat(12, 16 << 12, seed=3).with_weights(rb.WEIGHTS_UNIFORM, seed=4,
                                                             lo=0.0, hi=0.3)
    dg = rb.DeviceGraph(ctx, g, "IC")
    r = dg.autotune(seed=5, pilot=512)
    assert 0 <= r["choice"] < len(dg.TUNE_NAMES) and len(r["ms"]) == len(dg.TUNE_NAMES)
    p = rb.Pool(dg)
    p.sample(1500, seed=9)  # RIP_SAMPLER_AUTO: the tuned configuration
    thr = O.pack("IC", g.index, g.weights)
    ooff, ovtx, _ = O.sample("IC", g.n, g.index, g.src, thr, 9, 0, 1500)
    off, vtx = p.export()
    assert np.array_equal(off, ooff) and np.array_equal(vtx, ovtx)
    p.close()
    dg.close()
    lt = rb.DeviceGraph(ctx, lt_graph(11), "LT")
    assert lt.autotune(seed=1)["choice"] == 0
    lt.close()


def test_server_suspends_under_memory_pressure_and_answers_stay_exact():
    # a context whose budget fits one of these queries' pools at a time: the
    # server must suspend one (its pool freed, restarted later) rather than
    # fail it, and every answer must equal the query alone
    small = rb.Context(0, hbm_budget=600 << 20)
    g = lt_graph(16, 8, seed=31)
    dg = rb.DeviceGraph(small, g, "LT")
    specs = [(40, 0.12, 1), (30, 0.12, 2), (20, 0.2, 3)]
    alone_res = []
    for k, e, s in specs:
        p = rb.Pool(dg)
        seeds, rec = p.imm(k, e, seed=s, tiebreak=rb.TIE_LOWEST_ID)
        alone_res.append((seeds.tolist(), rec.theta))
        p.close()
    srv = rb.Server(small, max_active=3)
    qs = [srv.submit(rb.Query(dg, k, e, seed=s)) for k, e, s in specs]
    srv.drain()
    for q, (seeds, theta) in zip(qs, alone_res):
        assert q.done and q.status == 0
        assert q.seeds.tolist() == seeds and q.record.theta == theta
    srv.close()
    dg.close()
    small.close()


def test_server_slot_reuse_across_k(ctx, graphs):
    # one slot serves k = 10, then a larger k (its buffers grow), then k = 10
    # again: the round captured for the first k must not reuse the old buffers
    hs, dev = graphs
    srv = rb.Server(ctx, max_active=1)
    specs = [("lt12", 10, 0.5, 1), ("lt12", 60, 0.5, 1), ("lt12", 10, 0.4, 1),
             ("ic12", 10, 0.5, 0), ("ic12", 70, 0.5, 0), ("ic12", 10, 0.5, 0)]
    qs = [srv.submit(rb.Query(dev[n], k, e, seed=s)) for n, k, e, s in specs]
    srv.drain()
    for (n, k, e, s), q in zip(specs, qs):
        assert q.done and q.status == 0
        ref, rec = alone(dev, n, k, e, s, rb.TIE_LOWEST_ID)
        assert q.seeds.tolist() == ref.tolist(), (n, k, e)
    srv.close()


def test_server_index_segments_and_merge(ctx, graphs):
    # one pool grown by many later queries in turn (each needs more sets than
    # the last): its vertex -> sets index gains a segment per growth step and
    # is merged back into one past the segment limit; answers stay exact
    hs, dev = graphs
    srv = rb.Server(ctx, max_active=1)
    specs = [("lt13", 5 + 4 * i, 0.5 - 0.03 * i, 7) for i in range(12)]
    qs = [srv.submit(rb.Query(dev[n], k, e, seed=s)) for n, k, e, s in specs]
    srv.drain()
    for (n, k, e, s), q in zip(specs, qs):
        assert q.done and q.status == 0
        ref, rec = alone(dev, n, k, e, s, rb.TIE_LOWEST_ID)
        assert q.seeds.tolist() == ref.tolist(), (k, e)
        assert q.record.theta == rec.theta
    srv.close()
