"""Concurrent queries on one device: IMMs run from several host threads, each
with its own context (graph copy and pool), return exactly what each query
returns when run alone.  bench.py times its IMM workloads this way (a query's
reference-heap selection waits on the host while another query's kernels use
the GPU), so the contexts must share nothing but the device."""
import threading

import numpy as np
import pytest

import ripples_b200 as rb

pytestmark = pytest.mark.gpu


def graphs():
    ic = rb.HostGraph.rmat(13, 8 << 13, seed=3).with_weights(rb.WEIGHTS_WC)
    lt = rb.HostGraph.rmat(13, 8 << 13, seed=4).with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=5)
    return [("IC", ic), ("LT", lt)]


@pytest.mark.parametrize("model,g", graphs(), ids=["IC", "LT"])
def test_concurrent_contexts_match_alone(model, g):
    queries = [(20, 0.3, 100 + i) for i in range(8)]
    # alone: one context, one query after another
    alone = []
    cx = rb.Context(0)
    dg = rb.DeviceGraph(cx, g, model)
    pool = rb.Pool(dg)
    for k, eps, seed in queries:
        pool.clear()
        seeds, rec = pool.imm(k, eps, 1.0, seed=seed)
        alone.append((seeds.tolist(), rec.theta, rec.total_sets, rec.f))
    cx.close()
    # concurrent: four threads, a context each, two queries each
    n_clients = 4
    got = [None] * len(queries)
    errors = []

    def client(j):
        try:
            c = rb.Context(0)
            d = rb.DeviceGraph(c, g, model)
            p = rb.Pool(d)
            for i in range(j, len(queries), n_clients):
                k, eps, seed = queries[i]
                p.clear()
                seeds, rec = p.imm(k, eps, 1.0, seed=seed)
                got[i] = (seeds.tolist(), rec.theta, rec.total_sets, rec.f)
            c.close()
        except Exception as exc:  # reported after the join
            errors.append(repr(exc))

    threads = [threading.Thread(target=client, args=(j,)) for j in range(n_clients)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    assert got == alone
    # the queries differ from each other (the comparison is not vacuous)
    assert len({tuple(a[0]) for a in alone}) > 1
    assert np.all([a[1] > 0 for a in alone])
