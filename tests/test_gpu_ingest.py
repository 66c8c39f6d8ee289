"""Graph ingestion on the device (rip_graph_from_edges): a TSV file's edge
list renumbered, transposed into the backward CSR and packed on the GPU.  The
result must equal the host reader's graph (rip_read_tsv, pinned to the
reference's loader and GraphBwd constructor in tests/test_host.py) uploaded
with rip_graph_upload -- offsets, in-edge sources, packed thresholds and the id
map -- and the reference loader's own structure (include/ripples/loaders.h:
138-196, graph.h:506-620), and sampling from it must give the same sets."""
import numpy as np
import pytest

import ripples_b200 as rb
from conftest import GOLDEN
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _tsv(tmp_path, name, weighted, seed=5, n_lines=20000, span=6000):
    rng = np.random.default_rng(seed)
    lines = ["# edge list", "% comment"]
    for i in range(n_lines):
        a, b = rng.integers(3, span, size=2)
        lines.append(f"{a}\t{b}\t{rng.random() * 0.3:.6f}" if weighted else f"{a}\t{b}")
        if i % 997 == 0:
            lines.append(lines[-1])  # parallel edges
    p = tmp_path / name
    p.write_text("\n".join(lines) + "\n")
    return str(p)


@pytest.mark.parametrize("weighted,undirected,renumber,model",
                         [(1, 0, 1, "IC"), (1, 1, 1, "IC"), (0, 0, 0, "IC"), (0, 1, 1, "LT"),
                          (1, 0, 0, "LT")])
def test_device_build_equals_host_reader(ctx, tmp_path, weighted, undirected, renumber, model):
    p = _tsv(tmp_path, "g.tsv", weighted)
    s, d, w = rb.HostGraph.read_tsv_edges(p, weighted=bool(weighted), undirected=bool(undirected),
                                          model=model)
    g, rmap = rb.HostGraph.read_tsv(p, weighted=bool(weighted), undirected=bool(undirected),
                                    renumber=bool(renumber), model=model)
    dev = rb.DeviceGraph.from_edges(ctx, s, d, w, model, renumber=bool(renumber))
    ref = rb.DeviceGraph(ctx, g, model)
    try:
        assert dev.n == g.n and dev.m == g.m
        idx, src = dev.export()
        assert np.array_equal(idx, g.index) and np.array_equal(src, g.src)
        assert np.array_equal(dev.thresholds(), ref.thresholds())
        assert np.array_equal(dev.id_map(), rmap)
        # the same graph samples the same sets
        pa, pb = rb.Pool(dev), rb.Pool(ref)
        pa.sample(2000, seed=9)
        pb.sample(2000, seed=9)
        oa, va = pa.export()
        ob, vb = pb.export()
        assert np.array_equal(oa, ob) and np.array_equal(va, vb)
        pa.close()
        pb.close()
    finally:
        dev.close()
        ref.close()


def test_device_build_matches_reference_loader(ctx, tmp_path):
    # karate (the reference's test graph) and a larger random file, as the
    # reference's sequential loader + GraphBwd constructor build them
    if O.reference() is None:
        pytest.skip("oracle/_ref not built")
    for p in (f"{GOLDEN}/karate.tsv", _tsv(tmp_path, "u.tsv", weighted=0, seed=11)):
        for undirected in (0, 1):
            n, idx, src, w, rmap = O.ref_load_tsv(p, undirected, False, True)
            s, d, ww = rb.HostGraph.read_tsv_edges(p, undirected=bool(undirected))
            dev = rb.DeviceGraph.from_edges(ctx, s, d, ww, "IC")
            try:
                didx, dsrc = dev.export()
                assert dev.n == n and np.array_equal(didx, idx)
                assert np.array_equal(dev.id_map(), rmap)
                for v in range(n):  # the reference fills in-lists in parallel
                    assert sorted(src[idx[v]:idx[v + 1]].tolist()) == \
                        dsrc[didx[v]:didx[v + 1]].tolist()
            finally:
                dev.close()


def test_device_build_rejects_bad_input(ctx):
    with pytest.raises(rb.RipError):
        rb.DeviceGraph.from_edges(ctx, [], [], [], "IC")
