"""Generates the golden fixtures under tests/golden/ from the REFERENCE itself.

Run in a container where the reference tree is available and
``make -f oracle/ref.mk`` has built oracle/_ref/ (the reference's selection,
theta math and samplers compiled from its own sources):

    python tests/golden/make_golden.py

Outputs (small, committed):
  selection_cases.npz   random RRR-set lists (tie-heavy) with the seeds and f
                        returned by the reference's FindMostInfluentialSet
                        (omp_parallel_tag, 4 threads, and sequential_tag)
  theta_values.json     reference ThetaPrime / InvThetaPrime / Theta /
                        logBinomial on a parameter grid
  kat_counting.json     the counting / update known-answer vectors of the
                        reference's test/cuda_find_most_influential.cc:56-167
  sampler_reference.npz per-vertex occurrence counts and set sizes of the
                        reference's sequential IC / LT samplers on fixed graphs
                        (trng interface shim as the random stream)
  spread_reference.json mean IC / LT spread of fixed seed sets measured by
                        the reference's simulator (ripples::simulate)
  opimc_values.json     the reference's OPIM-C sample sizes and bounds on a
                        grid (include/ripples/opimc.h:60-98), floats as bits
The karate graph (karate.tsv, 78 edges) is the reference's
test-data/karate.tsv / test/rrr_set_generation.cc:63-79 edge list.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
import ripples_b200 as rb  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def selection_cases():
    rng = np.random.default_rng(20241203)
    cases = []
    for i in range(60):
        n = int(rng.integers(8, 80))
        S = int(rng.integers(1, 600))
        k = int(rng.integers(1, 15))
        maxsz = int(rng.integers(1, 9))
        sets = [np.sort(rng.choice(n, size=int(rng.integers(1, min(n, maxsz) + 1)),
                                   replace=False)) for _ in range(S)]
        cases.append((n, sets, k))
    # larger cases: sets sampled by the oracle on a small R-MAT graph
    for scale, nsets, k in [(10, 3000, 25), (11, 6000, 40)]:
        g = rb.HostGraph.rmat(scale, 8 << scale, seed=scale).with_weights(
            rb.WEIGHTS_UNIFORM, seed=2, lo=0.0, hi=0.2)
        thr = O.pack("IC", g.index, g.weights)
        off, vtx, _ = O.sample("IC", g.n, g.index, g.src, thr, 11, 0, nsets)
        sets = [vtx[off[i]:off[i + 1]] for i in range(nsets)]
        cases.append((g.n, sets, k))
    arrays = {}
    for i, (n, sets, k) in enumerate(cases):
        off = np.zeros(len(sets) + 1, np.uint64)
        off[1:] = np.cumsum([len(s) for s in sets])
        vtx = np.concatenate(sets).astype(np.uint32)
        f_omp, s_omp = O.ref_select(n, off, vtx, k, omp=True, threads=4)
        f_seq, s_seq = O.ref_select(n, off, vtx, k, omp=False)
        assert list(s_omp) == list(s_seq) and f_omp == f_seq, i
        arrays[f"c{i}_meta"] = np.array([n, k], np.uint64)
        arrays[f"c{i}_off"] = off
        arrays[f"c{i}_vtx"] = vtx
        arrays[f"c{i}_seeds"] = s_omp.astype(np.uint32)
        arrays[f"c{i}_f"] = np.array([f_omp], np.float64)
    arrays["num_cases"] = np.array([len(cases)], np.uint64)
    np.savez_compressed(os.path.join(OUT, "selection_cases.npz"), **arrays)


def theta_values():
    R = O.reference()
    rows = []
    for n in [34, 1000, 1 << 14, 1 << 20, 1 << 24]:
        for k in [1, 20, 50, 100, 500]:
            for eps in [0.5, 0.3, 0.13]:
                l = 1.0 * (1 + 1 / np.log2(n))
                ep = 1.4142135623730951 * eps
                for x in range(1, int(np.log2(n)) + 1):
                    rows.append({"kind": "theta_prime", "x": x, "eps_prime": ep, "l": l,
                                 "k": k, "n": n,
                                 "value": int(R.ref_theta_prime(x, ep, l, k, n))})
                for rr in [1, 100, 12345, 10 ** 6]:
                    rows.append({"kind": "inv_theta_prime", "x": rr, "eps_prime": ep, "l": l,
                                 "k": k, "n": n,
                                 "value": int(R.ref_inv_theta_prime(rr, ep, l, k, n))})
                for lb in [0.0, 1.0, 17.5, 1234.5678, n / 3.0]:
                    rows.append({"kind": "theta", "eps": eps, "l": l, "k": k, "lb": lb, "n": n,
                                 "value": int(R.ref_theta(eps, l, k, lb, n))})
            rows.append({"kind": "log_binomial", "n": n, "k": min(k, n // 2),
                         "value": float(R.ref_log_binomial(n, min(k, n // 2)))})
    with open(os.path.join(OUT, "theta_values.json"), "w") as fh:
        json.dump(rows, fh)


def kat_counting():
    # test/cuda_find_most_influential.cc:56-77 builds 1100 sets, but sizes its
    # device buffers for 2000 + 66*2 + 33*3 = 2231 elements (:85-87) and copies
    # only that many: the loop makes 34 sets {3,4,5}, so the last set (i = 99)
    # never reaches the device.  Its expected counts (566 / 33 / 566) are those
    # of the first 1099 sets, which is what this fixture holds.
    sets = [[2, 3] if i % 2 else [2, 5] for i in range(1000)]
    for i in range(100):
        sets.append([[3, 4, 5], [1, 3], [1, 5]][i % 3])
    assert sum(len(s) for s in sets[:-1]) == 2000 + 66 * 2 + 33 * 3
    sets = sets[:-1]
    kat = {
        "n": 6,
        "sets": sets,
        "counts": [0, 66, 1000, 566, 33, 566],                     # :101-106
        "after_seed_2": [0, 66, 0, 66, 33, 66],                    # :123-128
        "mask_after_2": [1] * 1000 + [0] * 99,                     # :116-121
        "after_seed_1": [0, 0, 0, 33, 33, 33],                     # :159-164
        "mask_after_1_tail": [[0, 1, 1][i % 3] for i in range(99)],  # :140-157
    }
    with open(os.path.join(OUT, "kat_counting.json"), "w") as fh:
        json.dump(kat, fh)


def sampler_reference():
    """Reference sequential samplers on two fixed graphs, for the
    distributional comparison (per-vertex frequencies, mean set size)."""
    out = {}
    tmp = tempfile.mkdtemp()
    graphs = {
        "karate_ic": (karate_graph(), "IC"),
        "rmat10_ic": (rb.HostGraph.rmat(10, 8 << 10, seed=3).with_weights(
            rb.WEIGHTS_UNIFORM, seed=4, lo=0.0, hi=0.3), "IC"),
        "rmat10_lt": (rb.HostGraph.rmat(10, 8 << 10, seed=5).with_weights(
            rb.WEIGHTS_LT_NORMALIZED, seed=6), "LT"),
        # weighted cascade p = 1/indeg, the 2^24 IC workload's weight model
        "rmat10_wc": (rb.HostGraph.rmat(10, 16 << 10, seed=9).with_weights(rb.WEIGHTS_WC),
                      "IC"),
    }
    for name, (g, model) in graphs.items():
        path = os.path.join(tmp, name + ".bin")
        g.write_binary(path, backward=True)
        nsets = 200000
        off, vtx = O.ref_sample(path, model, nsets, seed=0)
        freq = np.bincount(vtx, minlength=g.n).astype(np.uint64)
        sizes = np.diff(off).astype(np.uint64)
        out[name + "_freq"] = freq
        out[name + "_size_hist"] = np.bincount(sizes.astype(np.int64)).astype(np.uint64)
        out[name + "_nsets"] = np.array([nsets], np.uint64)
        out[name + "_index"] = g.index
        out[name + "_src"] = g.src
        out[name + "_w"] = g.weights
    np.savez_compressed(os.path.join(OUT, "sampler_reference.npz"), **out)


# Weighted cascade on R-MAT 2^16 (32 draws per vertex), the 2^24 IC
# workload's weight model at a size where 2 M reference sets make the 1% mean
# size bound a 3-sigma test.  The graph is rebuilt from these parameters by the
# tests (oracle.rmat_graph), so the fixture holds only the reference's counts.
WC16 = dict(scale=16, draws=32 << 16, seed=0, nsets=2_000_000, sampler_seed=0)


def sampler_reference_wc16():
    n, idx, src, w = O.rmat_graph(WC16["scale"], WC16["draws"], seed=WC16["seed"],
                                  weights="wc")
    tmp = tempfile.mkdtemp()
    path = os.path.join(tmp, "wc16.bin")
    O.write_binary(path, n, idx, src, w)
    off, vtx = O.ref_sample(path, "IC", WC16["nsets"], seed=WC16["sampler_seed"])
    sizes = np.diff(off).astype(np.int64)
    np.savez_compressed(os.path.join(OUT, "sampler_reference_wc16.npz"),
                        freq=np.bincount(vtx, minlength=n).astype(np.uint64),
                        size_hist=np.bincount(sizes).astype(np.uint64),
                        nsets=np.array([WC16["nsets"]], np.uint64),
                        params=np.array([WC16["scale"], WC16["draws"], WC16["seed"]],
                                        np.uint64))


SPREAD_CASES = [
    # name, model, graph builder arguments, seed choice, replicas
    dict(name="karate_ic", model="IC", graph="karate", seeds="top2", replicas=100000),
    dict(name="rmat12_ic", model="IC", graph=dict(scale=12, draws=8 << 12, seed=7, wseed=8,
                                                  hi=0.2),
         seeds="top10", replicas=20000),
    dict(name="rmat14_ic", model="IC", graph=dict(scale=14, draws=1 << 18, seed=0, wseed=1,
                                                  hi=0.1),
         seeds="top20", replicas=5000),
    dict(name="karate_lt", model="LT", graph="karate", seeds="top2", replicas=50000),
    dict(name="rmat10_lt", model="LT", graph=dict(scale=10, draws=8 << 10, seed=7, wseed=8),
         seeds="top10", replicas=5000),
    dict(name="rmat12_lt", model="LT", graph=dict(scale=12, draws=8 << 12, seed=5, wseed=6),
         seeds="top10", replicas=12000),
]


def spread_graph(case) -> "rb.HostGraph":
    lt = case.get("model", "IC") == "LT"
    if case["graph"] == "karate":
        g = karate_graph()
        return g.with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=9) if lt else g
    p = case["graph"]
    g = rb.HostGraph.rmat(p["scale"], p["draws"], seed=p["seed"])
    if lt:
        return g.with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=p["wseed"])
    return g.with_weights(rb.WEIGHTS_UNIFORM, seed=p["wseed"], lo=0.0, hi=p["hi"])


def spread_seeds(g, choice) -> np.ndarray:
    """The `choice` = "topK" vertices of largest out-degree (ties: lower id)."""
    k = int(choice[3:])
    outdeg = np.bincount(g.src, minlength=g.n)
    return np.lexsort((np.arange(g.n), -outdeg))[:k].astype(np.uint32)


def spread_reference():
    """Mean IC / LT spread of fixed seed sets measured by the reference's own
    simulator (ripples::simulate, include/ripples/diffusion_simulation.h:73-178,
    driven as tools/simulator.cc does), for pinning the forward-spread
    restatements."""
    tmp = tempfile.mkdtemp()
    R = O.reference()
    rows = []
    for case in SPREAD_CASES:
        g = spread_graph(case)
        seeds = spread_seeds(g, case["seeds"])
        path = os.path.join(tmp, case["name"] + "_fwd.bin")
        g.write_binary(path, backward=False)
        spread = R.ref_simulate(path.encode(), 0 if case["model"] == "IC" else 1,
                                seeds.ctypes.data, len(seeds), case["replicas"], 0)
        rows.append(dict(case, seeds_list=[int(x) for x in seeds], spread=spread))
    with open(os.path.join(OUT, "spread_reference.json"), "w") as fh:
        json.dump(rows, fh, indent=1)


def opimc_values():
    """The reference's OPIM-C arithmetic (include/ripples/opimc.h:60-98) on a
    grid: theta_max, theta_0 and the two bounds (floats stored bit for bit)."""
    import itertools
    import struct
    R = O.reference()
    fbits = lambda x: struct.unpack("<I", struct.pack("<f", x))[0]
    rows = {"theta": [], "bounds": []}
    for n, eps, k, delta in itertools.product([34, 1000, 16384, 1 << 20, 1 << 24, 3000017],
                                              [0.05, 0.1, 0.13, 0.3, 0.5], [1, 5, 50, 100, 500],
                                              [0.01, 1e-3, 1.0 / 16384]):
        rows["theta"].append([n, fbits(eps), k, fbits(delta),
                              int(R.ref_opimc_theta_max(n, eps, k, delta)),
                              int(R.ref_opimc_theta_zero(n, eps, k, delta))])
    rng = np.random.default_rng(3)
    for _ in range(2000):
        n = int(rng.integers(10, 1 << 24))
        theta = int(rng.integers(1, 10 ** 7))
        cov = int(rng.integers(0, theta + 1))
        d = float(rng.choice([0.01, 0.001, 1e-4, 0.0333]))
        rows["bounds"].append([cov, fbits(d), n, theta,
                               fbits(R.ref_opimc_lower_bound(cov, d, n, theta)),
                               fbits(R.ref_opimc_upper_bound(cov, d, n, theta))])
    with open(os.path.join(OUT, "opimc_values.json"), "w") as fh:
        json.dump(rows, fh)


def karate_graph() -> "rb.HostGraph":
    e = np.loadtxt(os.path.join(OUT, "karate.tsv"), dtype=np.float64)
    src = e[:, 0].astype(np.int64) - 1  # 1-based ids in the file
    dst = e[:, 1].astype(np.int64) - 1
    return rb.HostGraph.from_edges(34, src, dst, e[:, 2].astype(np.float32))


if __name__ == "__main__":
    assert O.reference() is not None, "build oracle/_ref first: make -f oracle/ref.mk"
    selection_cases()
    theta_values()
    kat_counting()
    sampler_reference()
    sampler_reference_wc16()
    spread_reference()
    opimc_values()
    print("golden fixtures written to", OUT)
