"""Host-side product logic (no GPU): the C ABI library loads and exports every
declared symbol; theta math equals the reference's; graph construction helpers
are deterministic and write the reference's binary format."""
import ctypes
import os
import re
import struct

import numpy as np
import pytest

import ripples_b200 as rb
from ripples_b200 import _lib
from conftest import ROOT


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "ripples_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(rip_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    so = ctypes.CDLL(_lib.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(so, s)]
    assert not missing, missing
    # and the Python binding declares a signature for each of them
    assert set(syms) <= set(_lib.SIGNATURES), set(syms) - set(_lib.SIGNATURES)


def test_library_is_sm100a_only():
    assert "sm_100a" in rb.library_version()


def test_theta_math_matches_reference(golden_theta):
    for r in golden_theta:
        if r["kind"] == "theta_prime":
            assert rb.theta_prime(r["x"], r["eps_prime"], r["l"], r["k"], r["n"]) == r["value"]
        elif r["kind"] == "inv_theta_prime":
            assert rb.inv_theta_prime(r["x"], r["eps_prime"], r["l"], r["k"], r["n"]) == r["value"]
        elif r["kind"] == "theta":
            assert rb.theta(r["eps"], r["l"], r["k"], r["lb"], r["n"]) == r["value"]
        else:
            assert rb.log_binomial(r["n"], r["k"]) == r["value"]


def test_rmat_deterministic_and_clean():
    a = rb.HostGraph.rmat(12, 1 << 16, seed=5)
    b = rb.HostGraph.rmat(12, 1 << 16, seed=5)
    c = rb.HostGraph.rmat(12, 1 << 16, seed=6)
    assert np.array_equal(a.index, b.index) and np.array_equal(a.src, b.src)
    assert not np.array_equal(a.src, c.src)
    assert a.n == 4096 and a.index[0] == 0 and a.index[-1] == a.m
    assert 0 < a.m <= 1 << 16
    dst = np.repeat(np.arange(a.n), np.diff(a.index).astype(np.int64))
    assert np.all(a.src != dst)  # no self loops
    key = dst.astype(np.uint64) << np.uint64(32) | a.src.astype(np.uint64)
    assert np.all(np.diff(key.astype(np.int64)) > 0)  # sorted by (dst, src), no duplicates
    # R-MAT skew: vertex 0 (all-"a" quadrant) is the heaviest source
    out_deg = np.bincount(a.src, minlength=a.n)
    assert out_deg.argmax() == 0


def test_erdos_renyi():
    g = rb.HostGraph.erdos_renyi(1000, 20000, seed=1)
    assert g.n == 1000 and 19000 < g.m <= 20000
    deg = np.diff(g.index)
    assert deg.max() < 60  # no skew


def test_weight_models():
    g = rb.HostGraph.rmat(10, 1 << 14, seed=2)
    u = g.with_weights(rb.WEIGHTS_UNIFORM, seed=1, lo=0.0, hi=0.1).weights
    assert u.min() >= 0 and u.max() < 0.1 and abs(u.mean() - 0.05) < 0.005
    lt = g.with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=1).weights
    sums = np.add.reduceat(lt.astype(np.float64), g.index[:-1].astype(np.int64)[np.diff(g.index) > 0])
    assert np.allclose(sums, 1.0, atol=1e-5)
    wc = g.with_weights(rb.WEIGHTS_WC).weights
    deg = np.diff(g.index).astype(np.int64)
    assert np.allclose(wc, np.repeat(1.0 / np.maximum(deg, 1), deg).astype(np.float32))


def test_binary_format_layout(tmp_path):
    g = rb.HostGraph.rmat(8, 2000, seed=3).with_weights(rb.WEIGHTS_UNIFORM, seed=1, lo=0, hi=1)
    p = str(tmp_path / "g.bin")
    g.write_binary(p, backward=True)
    raw = open(p, "rb").read()
    hdr = struct.unpack("<5Q", raw[:40])
    assert hdr == (0xC0FFEE, 0xA1CCAC0F, 32, g.n, g.m)
    off = 40
    rmap = np.frombuffer(raw, np.uint32, g.n, off); off += 4 * g.n
    idx = np.frombuffer(raw, np.uint64, g.n + 1, off); off += 8 * (g.n + 1)
    src = np.frombuffer(raw, np.uint32, g.m, off); off += 4 * g.m
    w = np.frombuffer(raw, np.float32, g.m, off); off += 4 * g.m
    assert off == len(raw)
    assert np.array_equal(rmap, np.arange(g.n)) and np.array_equal(idx, g.index)
    assert np.array_equal(src, g.src) and np.array_equal(w, g.weights)
    pf = str(tmp_path / "f.bin")
    g.write_binary(pf, backward=False)
    hdr = struct.unpack("<5Q", open(pf, "rb").read()[:40])
    assert hdr[1] == 0xF0CACC1A


def test_binary_loads_in_reference(tmp_path):
    from oracle import oracle as O
    R = O.reference()
    if R is None:
        pytest.skip("oracle/_ref not built")
    g = rb.HostGraph.rmat(9, 4000, seed=4).with_weights(rb.WEIGHTS_UNIFORM, seed=1, lo=0, hi=1)
    p = str(tmp_path / "g.bin")
    g.write_binary(p)
    h = R.ref_graph_load(p.encode())
    assert R.ref_graph_nodes(h) == g.n and R.ref_graph_edges(h) == g.m
    R.ref_graph_free(h)


def test_context_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(rb.RipError):
        rb.Context(0)


def test_json_log_keys():
    CFG = rb.IMMConfiguration(k=5, epsilon=0.5, diffusionModel="IC")
    rec = rb.IMMExecutionRecord(Theta=10, ThetaPrimeDeltas=[3])
    e = rec.experiment(CFG, [1, 2])
    for key in ["Algorithm", "Input", "Output", "DiffusionModel", "Epsilon", "K", "L",
                "NumThreads", "NumWalkWorkers", "NumCPUTeams", "NumGPUWalkWorkers",
                "PauseThreshold", "Total", "ThetaPrimeDeltas", "ThetaEstimation",
                "ThetaEstimationGenerateRRR", "ThetaEstimationMostInfluential", "Theta",
                "Counting", "Pivoting", "Microbenchmarking", "CPUBatchSize", "GPUBatchSize",
                "RRRSetSizeBytes", "GenerateRRRSets", "FindMostInfluentialSet", "Seeds"]:
        assert key in e


@pytest.mark.parametrize("n,max_count,seed", [(1, 3, 0), (2, 1, 1), (37, 2, 2), (5000, 3, 3),
                                              (1 << 20, 5, 4), ((1 << 20) + 12345, 1000, 5)])
def test_parallel_heap_is_libstdcxx_make_heap(n, max_count, seed):
    """The selection heap is built level-parallel; it must equal
    std::make_heap element for element (the reference's tie-break depends on
    the exact heap layout), including with heavy ties."""
    assert _lib.lib.rip_selftest_heap(n, max_count, seed) == 1


# ---- graph input files (rip_read_tsv / rip_read_binary) ---------------------

def _write(path, text):
    with open(path, "w") as fh:
        fh.write(text)
    return str(path)


@pytest.mark.parametrize("undirected,renumber,lt", [(u, r, l) for u in (0, 1) for r in (0, 1)
                                                    for l in (0, 1)])
def test_read_tsv_structure_matches_reference_loader(tmp_path, undirected, renumber, lt):
    # The graph the reference's sequential loader and GraphBwd constructor
    # build from the same file: n, offsets, id map and each vertex's in-edge
    # sources (the reference fills in-lists in parallel; here they are sorted
    # by source id).  LT generated weights: per-source sums below 1 on both
    # sides (the "not taking" mass).
    from oracle import oracle as O
    if O.reference() is None:
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(7)
    lines = ["# header", "% comment"]
    for i in range(2000):
        s, t = rng.integers(0, 1500, size=2)
        lines.append(f"{s}\t{t}")
        if i % 101 == 0:
            lines.append("")
    p = _write(tmp_path / "g.tsv", "\n".join(lines) + "\n")
    n, idx, src, w, rmap = O.ref_load_tsv(p, undirected, lt, renumber)
    g, rmap2 = rb.HostGraph.read_tsv(p, undirected=bool(undirected), renumber=bool(renumber),
                                     model="LT" if lt else "IC")
    assert n == g.n and np.array_equal(idx, g.index) and np.array_equal(rmap, rmap2)
    for v in range(n):
        assert sorted(src[idx[v]:idx[v + 1]].tolist()) == \
            g.src[g.index[v]:g.index[v + 1]].tolist()
    assert (g.weights >= 0).all() and (g.weights < 1).all()
    if lt:
        for s_, w_ in ((src, w), (g.src, g.weights)):
            out = np.zeros(n)
            np.add.at(out, s_, w_)
            assert out.max() < 1.0 + 1e-6


def test_read_tsv_weighted_options(tmp_path):
    p = _write(tmp_path / "w.tsv", "# c\n10 20 0.5\n20 30 0.25\n\n% x\n50 10 0.75\n10 20 0.125\n")
    g, rmap = rb.HostGraph.read_tsv(p, weighted=True)
    assert g.n == 4 and rmap.tolist() == [10, 20, 30, 50]
    assert g.index.tolist() == [0, 1, 3, 4, 4]       # in-edges of 10, 20, 30, 50
    assert g.src.tolist() == [3, 0, 0, 1]            # by source id, duplicates kept
    assert g.weights.tolist() == [0.75, 0.5, 0.125, 0.25]
    g2, _ = rb.HostGraph.read_tsv(p, weighted=True, undirected=True)
    assert g2.m == 8
    for v in range(g2.n):  # the reverse edge carries the same weight
        for e in range(int(g2.index[v]), int(g2.index[v + 1])):
            u = int(g2.src[e])
            back = [float(g2.weights[f]) for f in range(int(g2.index[u]), int(g2.index[u + 1]))
                    if int(g2.src[f]) == v]
            assert float(g2.weights[e]) in back
    g3, rmap3 = rb.HostGraph.read_tsv(p, weighted=True, renumber=False, scale=0.5)
    assert g3.n == 51 and np.array_equal(rmap3, np.arange(51))
    assert sorted(g3.weights.tolist()) == [0.0625, 0.125, 0.25, 0.375]


def test_read_tsv_generated_weights_and_errors(tmp_path):
    p = _write(tmp_path / "u.tsv", "".join(f"{i} {(i * 7) % 50}\n" for i in range(200)))
    a, _ = rb.HostGraph.read_tsv(p)
    b, _ = rb.HostGraph.read_tsv(p)
    assert np.array_equal(a.weights, b.weights)   # one deterministic stream
    c, _ = rb.HostGraph.read_tsv(p, distribution="const", mean=0.3)
    assert np.allclose(c.weights, 0.3)
    d, _ = rb.HostGraph.read_tsv(p, distribution="normal", mean=0.4, variance=0.1)
    assert (d.weights >= 0).all() and (d.weights < 1).all()
    with pytest.raises(rb.RipError, match="cannot open"):
        rb.HostGraph.read_tsv(str(tmp_path / "missing.tsv"))
    with pytest.raises(rb.RipError, match="Unsupported distribution"):
        rb.HostGraph.read_tsv(p, distribution="pareto")
    with pytest.raises(rb.RipError, match="scale factor"):
        rb.HostGraph.read_tsv(p, scale=2.0)
    big = _write(tmp_path / "big.tsv", "1 2\n3 4294967295\n")
    with pytest.raises(rb.RipError, match="line 2"):
        rb.HostGraph.read_tsv(big)


def test_read_tsv_edges_is_the_readers_edge_list(tmp_path):
    # rip_read_tsv_edges stops before the Graph constructor: renumbering its
    # edges (sorted distinct ids) and ordering them by (destination, source),
    # stably, gives rip_read_tsv's CSR -- what rip_graph_from_edges does on the
    # device.
    rng = np.random.default_rng(3)
    lines = [f"{a}\t{b}\t{rng.random():.6f}" for a, b in rng.integers(5, 900, size=(1500, 2))]
    p = _write(tmp_path / "e.tsv", "# c\n" + "\n".join(lines) + "\n")
    for undirected in (False, True):
        s, d, w = rb.HostGraph.read_tsv_edges(p, weighted=True, undirected=undirected)
        g, rmap = rb.HostGraph.read_tsv(p, weighted=True, undirected=undirected)
        ids = np.unique(np.concatenate([s, d]))
        assert np.array_equal(ids, rmap)
        rs, rd = np.searchsorted(ids, s), np.searchsorted(ids, d)
        order = np.lexsort((rs, rd))  # stable: by destination, then source
        assert np.array_equal(rs[order].astype(np.uint32), g.src)
        assert np.array_equal(w[order], g.weights)
        assert np.array_equal(np.searchsorted(rd[order], np.arange(g.n + 1)), g.index)


def test_read_binary_round_trip_and_errors(tmp_path):
    g = rb.HostGraph.rmat(9, 4000, seed=4).with_weights(rb.WEIGHTS_UNIFORM, seed=1, lo=0, hi=1)
    p = str(tmp_path / "g.bin")
    g.write_binary(p)
    h, rmap = rb.HostGraph.read_binary(p)
    assert h.n == g.n and np.array_equal(rmap, np.arange(g.n))
    assert np.array_equal(h.index, g.index) and np.array_equal(h.src, g.src)
    assert np.array_equal(h.weights, g.weights)
    h2, _ = rb.HostGraph.read_binary(p, scale=0.5)
    assert np.array_equal(h2.weights, (g.weights * 0.5).astype(np.float32))
    raw = open(p, "rb").read()
    bad = str(tmp_path / "bad.bin")
    open(bad, "wb").write(b"\x00" * 8 + raw[8:])
    with pytest.raises(rb.RipError, match="endianess"):
        rb.HostGraph.read_binary(bad)
    open(bad, "wb").write(raw[: len(raw) - 12])
    with pytest.raises(rb.RipError, match="truncated"):
        rb.HostGraph.read_binary(bad)
    pf = str(tmp_path / "f.bin")
    g.write_binary(pf, backward=False)  # the forward direction is another format id
    with pytest.raises(rb.RipError, match="not compatible"):
        rb.HostGraph.read_binary(pf)


def test_opimc_arithmetic_matches_reference_golden():
    # theta_max, theta_0 and the two bounds of OPIM-C bit for bit against
    # the reference (include/ripples/opimc.h:60-98, golden grid).
    import json
    from conftest import GOLDEN
    with open(os.path.join(GOLDEN, "opimc_values.json")) as fh:
        rows = json.load(fh)
    f = lambda bits: struct.unpack("<f", struct.pack("<I", bits))[0]
    lib = _lib.lib
    for n, eps, k, delta, tmax, tzero in rows["theta"]:
        assert lib.rip_opimc_theta_max(n, f(eps), k, f(delta)) == tmax
        assert lib.rip_opimc_theta_zero(n, f(eps), k, f(delta)) == tzero
    bits = lambda x: struct.unpack("<I", struct.pack("<f", x))[0]
    for cov, d, n, theta, lo, up in rows["bounds"]:
        assert bits(lib.rip_opimc_lower_bound(cov, f(d), n, theta)) == lo
        assert bits(lib.rip_opimc_upper_bound(cov, f(d), n, theta)) == up


def test_transpose_and_forward_binary(tmp_path):
    # rip_transpose_csr gives the forward CSR HostGraph.forward() builds (and
    # back), and the forward binary format reads back as that CSR
    g = rb.HostGraph.rmat(9, 4000, seed=5).with_weights(rb.WEIGHTS_UNIFORM, seed=2, lo=0, hi=1)
    f = g.forward()
    t = g.transposed()
    assert np.array_equal(t.index, f.index) and np.array_equal(t.src, f.src)
    assert np.array_equal(t.weights, f.weights)
    back = t.transposed()
    assert np.array_equal(back.index, g.index) and np.array_equal(back.src, g.src)
    assert np.array_equal(back.weights, g.weights)
    p = str(tmp_path / "gf.bin")
    g.write_binary(p, backward=False)
    h, rmap = rb.HostGraph.read_binary(p, forward=True)
    assert np.array_equal(h.index, f.index) and np.array_equal(h.src, f.src)
    assert np.array_equal(h.weights, f.weights) and np.array_equal(rmap, np.arange(g.n))
    with pytest.raises(rb.RipError, match="not compatible"):
        rb.HostGraph.read_binary(p)  # a forward file is not a backward one
