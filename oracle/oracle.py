"""Python access to the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``oracle/liboracle.so`` (built from oracle/oracle.cpp by
oracle/Makefile) and, when present, ``oracle/_ref/libref_harness.so`` (the
reference's own selection / theta math / samplers compiled from its sources by
oracle/ref.mk).  Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline
leg of bench.py use this module; the product never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_harness.so")

P = ctypes.c_void_p
U32, U64, I32, I64, DBL = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_int64, ctypes.c_double


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load_oracle() -> ctypes.CDLL:
    if not os.path.exists(ORACLE_SO):
        build()
    L = ctypes.CDLL(ORACLE_SO)
    sig = {
        "orc_philox4x32_10": (None, [P, P, P]),
        "orc_root": (U32, [U64, U64, U32]),
        "orc_ic_coin": (U32, [U64, U64, U64]),
        "orc_lt_threshold": (U32, [U64, U64, U32]),
        "orc_pack_ic": (None, [P, U64, P]),
        "orc_pack_lt": (None, [P, U32, P, P]),
        "orc_sample": (P, [I32, U32, P, P, P, U64, U64, U64, P]),
        "orc_sample_ids": (P, [I32, U32, P, P, P, U64, P, U64]),
        "orc_rmat_csr": (I32, [U32, U64, DBL, DBL, DBL, U64, ctypes.POINTER(P), ctypes.POINTER(P),
                               ctypes.POINTER(U64)]),
        "orc_make_weights": (I32, [I32, U32, P, U64, DBL, DBL, P]),
        "orc_free": (None, [P]),
        "orc_spread_ic": (U64, [U32, P, P, P, P, U32, U64, U64, P, ctypes.POINTER(U64), P]),
        "orc_spread_lt": (U64, [U32, P, P, P, P, P, P, U32, U64, U64, P, P]),
        "orc_find_coverage": (U64, [U64, P, P, P, U32]),
        "orc_opimc": (U32, [I32, U32, P, P, P, U32, ctypes.c_float, ctypes.c_float, U64, I32, P,
                            ctypes.POINTER(U64), ctypes.POINTER(U32), P]),
        "orc_opimc_math": (None, [U64, ctypes.c_float, U64, ctypes.c_float, U64, U64, P, P]),
        "orc_pool_elements": (U64, [P]),
        "orc_pool_sets": (U64, [P]),
        "orc_pool_copy": (None, [P, P, P]),
        "orc_pool_free": (None, [P]),
        "orc_select": (U32, [U32, U64, P, P, U32, I32, P, P, ctypes.POINTER(DBL),
                             ctypes.POINTER(U64)]),
        "orc_theta_prime": (I64, [I64, DBL, DBL, U64, U64]),
        "orc_inv_theta_prime": (I64, [I64, DBL, DBL, U64, U64]),
        "orc_theta": (U64, [DBL, DBL, U64, DBL, U64]),
        "orc_log_binomial": (DBL, [U64, U64]),
        "orc_imm": (I32, [I32, U32, P, P, P, U32, DBL, U64, I32, P, ctypes.POINTER(U32),
                          ctypes.POINTER(U64), P, ctypes.POINTER(U32), ctypes.POINTER(DBL),
                          ctypes.POINTER(U64)]),
    }
    for k, (r, a) in sig.items():
        f = getattr(L, k)
        f.restype, f.argtypes = r, a
    return L


L = _load_oracle()


def philox(ctr, key):
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    L.orc_philox4x32_10(c, k, o)
    return list(o)


def root(seed: int, s: int, n: int) -> int:
    return int(L.orc_root(seed, s, n))


def pack(model: str, index: np.ndarray, weights: np.ndarray) -> np.ndarray:
    m = len(weights)
    thr = np.zeros(max(m, 1), dtype=np.uint32)
    w = np.ascontiguousarray(weights, dtype=np.float32)
    if model == "IC":
        L.orc_pack_ic(_ptr(w), m, _ptr(thr))
    else:
        idx = np.ascontiguousarray(index, dtype=np.uint64)
        L.orc_pack_lt(_ptr(idx), len(idx) - 1, _ptr(w), _ptr(thr))
    return thr[:m]


def sample(model: str, n: int, index: np.ndarray, src: np.ndarray, thr: np.ndarray,
           seed: int, first: int, count: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Sets [first, first+count) as CSR (offsets, vertices), each sorted, plus
    stats [expansions, in-edges read]."""
    idx = np.ascontiguousarray(index, dtype=np.uint64)
    s = np.ascontiguousarray(src, dtype=np.uint32)
    t = np.ascontiguousarray(thr, dtype=np.uint32)
    if s.size == 0:
        s = np.zeros(1, np.uint32)
        t = np.zeros(1, np.uint32)
    st = np.zeros(2, dtype=np.uint64)
    h = L.orc_sample(0 if model == "IC" else 1, n, _ptr(idx), _ptr(s), _ptr(t), seed, first,
                     count, _ptr(st))
    ns, ne = L.orc_pool_sets(h), L.orc_pool_elements(h)
    off = np.zeros(ns + 1, dtype=np.uint64)
    vtx = np.zeros(max(ne, 1), dtype=np.uint32)
    L.orc_pool_copy(h, _ptr(off), _ptr(vtx))
    L.orc_pool_free(h)
    return off, vtx[:ne], st


def sample_ids(model: str, n: int, index: np.ndarray, src: np.ndarray, thr: np.ndarray,
               seed: int, ids) -> Tuple[np.ndarray, np.ndarray]:
    """The sets with the listed ids as CSR (offsets, vertices), each sorted;
    drawn in parallel over the host threads."""
    idx = np.ascontiguousarray(index, dtype=np.uint64)
    s = np.ascontiguousarray(src, dtype=np.uint32)
    t = np.ascontiguousarray(thr, dtype=np.uint32)
    if s.size == 0:
        s = np.zeros(1, np.uint32)
        t = np.zeros(1, np.uint32)
    ids = np.ascontiguousarray(ids, dtype=np.uint64)
    h = L.orc_sample_ids(0 if model == "IC" else 1, n, _ptr(idx), _ptr(s), _ptr(t), seed,
                         _ptr(ids), len(ids))
    ns, ne = L.orc_pool_sets(h), L.orc_pool_elements(h)
    off = np.zeros(ns + 1, dtype=np.uint64)
    vtx = np.zeros(max(ne, 1), dtype=np.uint32)
    L.orc_pool_copy(h, _ptr(off), _ptr(vtx))
    L.orc_pool_free(h)
    return off, vtx[:ne]


WEIGHT_KINDS = {"uniform": 0, "lt_normalized": 1, "wc": 2}


def rmat_graph(scale: int, draws: int, a: float = 0.57, b: float = 0.19, c: float = 0.19,
               seed: int = 0, weights: str = "uniform", weight_seed: int = 1,
               lo: float = 0.0, hi: float = 0.1):
    """An R-MAT graph drawn as the library's host builder draws it, as the
    backward CSR (n, index u64[n+1], src u32[m], weights f32[m])."""
    pi, ps, m = P(), P(), U64()
    if L.orc_rmat_csr(scale, draws, a, b, c, seed, ctypes.byref(pi), ctypes.byref(ps),
                      ctypes.byref(m)) != 0:
        raise MemoryError("orc_rmat_csr failed")
    n, mm = 1 << scale, m.value
    try:
        index = np.ctypeslib.as_array(ctypes.cast(pi, ctypes.POINTER(U64)), (n + 1,)).copy()
        src = np.ctypeslib.as_array(ctypes.cast(ps, ctypes.POINTER(U32)), (max(mm, 1),))[:mm].copy()
    finally:
        L.orc_free(pi)
        L.orc_free(ps)
    w = np.zeros(max(mm, 1), dtype=np.float32)
    if L.orc_make_weights(WEIGHT_KINDS[weights], n, _ptr(index), weight_seed, lo, hi, _ptr(w)):
        raise ValueError("orc_make_weights failed")
    return n, index, src, w[:mm]


def write_binary(path: str, n: int, index, src, w) -> None:
    """The reference's binary graph format (include/ripples/graph.h:700-771),
    backward direction, float weights, identity id map."""
    m = len(src)
    with open(path, "wb") as fh:
        np.asarray([0xc0ffee, 0xa1ccac0f, 32, n, m], dtype=np.uint64).tofile(fh)
        np.arange(n, dtype=np.uint32).tofile(fh)
        np.ascontiguousarray(index, dtype=np.uint64).tofile(fh)
        np.ascontiguousarray(src, dtype=np.uint32).tofile(fh)
        np.ascontiguousarray(w, dtype=np.float32).tofile(fh)


def spread_ic(n: int, index: np.ndarray, dst: np.ndarray, thr: np.ndarray, seeds,
              replicas: int, seed: int = 0, with_edges: bool = False,
              with_levels: bool = False):
    """Forward IC spread over the forward CSR (index over sources, dst the
    out-edge targets, IC thresholds): (mean reached count, per-replica
    counts), plus the out-edges of the reached vertices summed over the
    replicas with ``with_edges``."""
    idx = np.ascontiguousarray(index, dtype=np.uint64)
    d = np.ascontiguousarray(dst, dtype=np.uint32)
    t = np.ascontiguousarray(thr, dtype=np.uint32)
    if d.size == 0:
        d = np.zeros(1, np.uint32)
        t = np.zeros(1, np.uint32)
    sd = np.ascontiguousarray(seeds, dtype=np.uint32)
    k = int(sd.size)
    if k == 0:
        sd = np.zeros(1, np.uint32)
    sizes = np.zeros(max(replicas, 1), dtype=np.uint32)
    edges = ctypes.c_uint64()
    levels = np.zeros(max(replicas, 1), dtype=np.uint32)
    total = L.orc_spread_ic(n, _ptr(idx), _ptr(d), _ptr(t), _ptr(sd), k, replicas, seed,
                            _ptr(sizes), ctypes.byref(edges), _ptr(levels))
    mean = total / replicas if replicas else 0.0
    out = [mean, sizes[:replicas]]
    if with_edges:
        out.append(edges.value)
    if with_levels:
        out.append(levels[:replicas])
    return tuple(out)


def spread_lt(g, seeds, replicas: int, seed: int = 0, with_levels: bool = False):
    """Forward LT spread (live-edge form) on backward HostGraph ``g`` with LT
    weights: (mean reached count, per-replica counts)."""
    f = g.forward()
    cum = pack("LT", g.index, g.weights)
    fi = np.ascontiguousarray(f.index, dtype=np.uint64)
    fd = np.ascontiguousarray(f.src, dtype=np.uint32)
    bi = np.ascontiguousarray(g.index, dtype=np.uint64)
    bs = np.ascontiguousarray(g.src, dtype=np.uint32)
    c = np.ascontiguousarray(cum, dtype=np.uint32)
    if fd.size == 0:
        fd, bs, c = (np.zeros(1, np.uint32) for _ in range(3))
    sd = np.ascontiguousarray(seeds, dtype=np.uint32)
    k = int(sd.size)
    if k == 0:
        sd = np.zeros(1, np.uint32)
    sizes = np.zeros(max(replicas, 1), dtype=np.uint32)
    levels = np.zeros(max(replicas, 1), dtype=np.uint32)
    total = L.orc_spread_lt(g.n, _ptr(fi), _ptr(fd), _ptr(bi), _ptr(bs), _ptr(c), _ptr(sd), k,
                            replicas, seed, _ptr(sizes), _ptr(levels))
    mean = total / replicas if replicas else 0.0
    if with_levels:
        return mean, sizes[:replicas], levels[:replicas]
    return mean, sizes[:replicas]


def opimc(model: str, n: int, index, src, thr, k: int, epsilon: float, delta: float,
          seed: int = 0, tiebreak: int = 0) -> dict:
    """OPIM-C (include/ripples/opimc.h:150-243) over the oracle: seeds, the
    final pool size, rounds, theta_0 and theta_max."""
    idx = np.ascontiguousarray(index, dtype=np.uint64)
    s = np.ascontiguousarray(src, dtype=np.uint32)
    t = np.ascontiguousarray(thr, dtype=np.uint32)
    seeds = np.zeros(max(k, 1), np.uint32)
    theta, rounds = ctypes.c_uint64(), ctypes.c_uint32()
    th = np.zeros(2, np.uint64)
    ns = L.orc_opimc(0 if model == "IC" else 1, n, _ptr(idx), _ptr(s), _ptr(t), k, epsilon, delta,
                     seed, tiebreak, _ptr(seeds), ctypes.byref(theta), ctypes.byref(rounds),
                     _ptr(th))
    return dict(seeds=seeds[:ns].tolist(), theta=theta.value, rounds=rounds.value,
                theta_zero=int(th[0]), theta_max=int(th[1]))


def opimc_math(n, epsilon, k, delta, coverage, theta):
    th = np.zeros(2, np.uint64)
    b = np.zeros(2, np.float32)
    L.orc_opimc_math(n, epsilon, k, delta, coverage, theta, _ptr(th), _ptr(b))
    return int(th[0]), int(th[1]), b


def find_coverage(offsets, vertices, seeds) -> int:
    """Sets holding at least one seed (OPIM-C's FindCoverage)."""
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    vtx = np.ascontiguousarray(vertices, dtype=np.uint32)
    sd = np.ascontiguousarray(seeds, dtype=np.uint32)
    if vtx.size == 0:
        vtx = np.zeros(1, np.uint32)
    k = int(sd.size)
    if k == 0:
        sd = np.zeros(1, np.uint32)
    return int(L.orc_find_coverage(len(off) - 1, _ptr(off), _ptr(vtx), _ptr(sd), k))


def ref_find_coverage(offsets, vertices, seeds) -> int:
    R = reference()
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    vtx = np.ascontiguousarray(vertices, dtype=np.uint32)
    sd = np.ascontiguousarray(seeds, dtype=np.uint32)
    if vtx.size == 0:
        vtx = np.zeros(1, np.uint32)
    return int(R.ref_find_coverage(len(off) - 1, _ptr(off), _ptr(vtx), _ptr(sd), int(len(seeds))))


def select(n: int, offsets: np.ndarray, vertices: np.ndarray, k: int, tiebreak: int = 0):
    """Greedy max coverage; returns (f, seeds, gains, uncovered).
    tiebreak 0 = reference CPU lazy heap, 1 = lowest id."""
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    vtx = np.ascontiguousarray(vertices, dtype=np.uint32)
    if vtx.size == 0:
        vtx = np.zeros(1, np.uint32)
    seeds = np.zeros(max(k, 1), dtype=np.uint32)
    gains = np.zeros(max(k, 1), dtype=np.uint64)
    f, unc = ctypes.c_double(), ctypes.c_uint64()
    ns = L.orc_select(n, len(off) - 1, _ptr(off), _ptr(vtx), k, tiebreak, _ptr(seeds),
                      _ptr(gains), ctypes.byref(f), ctypes.byref(unc))
    return f.value, seeds[:ns].copy(), gains[:ns].copy(), unc.value


def imm(model: str, n: int, index, src, thr, k: int, epsilon: float, seed: int = 0,
        tiebreak: int = 0) -> dict:
    idx = np.ascontiguousarray(index, dtype=np.uint64)
    s = np.ascontiguousarray(src, dtype=np.uint32)
    t = np.ascontiguousarray(thr, dtype=np.uint32)
    seeds = np.zeros(max(k, 1), dtype=np.uint32)
    deltas = np.zeros(64, dtype=np.uint64)
    ns, th, nr, ff, tot = ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint32(), \
        ctypes.c_double(), ctypes.c_uint64()
    L.orc_imm(0 if model == "IC" else 1, n, _ptr(idx), _ptr(s), _ptr(t), k, epsilon, seed,
              tiebreak, _ptr(seeds), ctypes.byref(ns), ctypes.byref(th), _ptr(deltas),
              ctypes.byref(nr), ctypes.byref(ff), ctypes.byref(tot))
    return {"seeds": seeds[:ns.value].tolist(), "theta": th.value,
            "deltas": deltas[:min(nr.value, 64)].tolist(), "f": ff.value,
            "total_sets": tot.value}


def theta_prime(x, eps_prime, l, k, n):
    return int(L.orc_theta_prime(x, eps_prime, l, k, n))


def inv_theta_prime(r, eps_prime, l, k, n):
    return int(L.orc_inv_theta_prime(r, eps_prime, l, k, n))


def theta(eps, l, k, lb, n):
    return int(L.orc_theta(eps, l, k, lb, n))


def log_binomial(n, k):
    return float(L.orc_log_binomial(n, k))


# ---- the reference itself (compiled from its sources), when available -------
_REF: Optional[ctypes.CDLL] = None


def reference() -> Optional[ctypes.CDLL]:
    """The reference harness, or None when oracle/_ref was not built."""
    global _REF
    if _REF is None and os.path.exists(REF_SO):
        R = ctypes.CDLL(REF_SO)
        sig = {
            "ref_select": (U32, [U32, U64, P, P, U32, I32, I32, P, ctypes.POINTER(DBL)]),
            "ref_theta_prime": (I64, [I64, DBL, DBL, U64, U64]),
            "ref_inv_theta_prime": (I64, [I64, DBL, DBL, U64, U64]),
            "ref_theta": (U64, [DBL, DBL, U64, DBL, U64]),
            "ref_log_binomial": (DBL, [U64, U64]),
            "ref_graph_load": (P, [ctypes.c_char_p]),
            "ref_graph_free": (None, [P]),
            "ref_graph_nodes": (U64, [P]),
            "ref_graph_edges": (U64, [P]),
            "ref_sample": (P, [P, I32, U64, U64, ctypes.POINTER(U64)]),
            "ref_pool_copy": (None, [P, P, P]),
            "ref_pool_free": (None, [P]),
            "ref_simulate": (DBL, [ctypes.c_char_p, I32, P, U32, U64, U64]),
            "ref_simulate_parallel": (DBL, [ctypes.c_char_p, I32, P, U32, U64]),
            "ref_simulate_levels": (DBL, [ctypes.c_char_p, I32, P, U32, U64, U64]),
            "ref_graph_load_tsv": (P, [ctypes.c_char_p, I32, I32, I32]),
            "ref_opimc_theta_max": (U64, [U64, ctypes.c_float, U64, ctypes.c_float]),
            "ref_opimc_theta_zero": (U64, [U64, ctypes.c_float, U64, ctypes.c_float]),
            "ref_opimc_lower_bound": (ctypes.c_float, [U64, ctypes.c_float, U64, U64]),
            "ref_opimc_upper_bound": (ctypes.c_float, [U64, ctypes.c_float, U64, U64]),
            "ref_find_coverage": (U64, [U64, P, P, P, U32]),
            "ref_graph_copy": (None, [P, P, P, P, P]),
            "ref_generate_parallel": (DBL, [P, U64, U64, ctypes.POINTER(U64)]),
            "ref_imm_sequential": (U32, [P, I32, U32, DBL, U64, P]),
        }
        for k, (r, a) in sig.items():
            f = getattr(R, k)
            f.restype, f.argtypes = r, a
        _REF = R
    return _REF


def ref_select(n: int, offsets, vertices, k: int, omp: bool = True, threads: int = 4):
    R = reference()
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    vtx = np.ascontiguousarray(vertices, dtype=np.uint32)
    if vtx.size == 0:
        vtx = np.zeros(1, np.uint32)
    seeds = np.zeros(max(k, 1) + 1, dtype=np.uint32)
    f = ctypes.c_double()
    ns = R.ref_select(n, len(off) - 1, _ptr(off), _ptr(vtx), k, 1 if omp else 0, threads,
                      _ptr(seeds), ctypes.byref(f))
    return f.value, seeds[:ns].copy()


def ref_load_tsv(path: str, undirected: bool, lt: bool, renumber: bool):
    """The reference's weighted TSV loader + GraphBwd: (n, index, src, w,
    reverse_map)."""
    R = reference()
    g = R.ref_graph_load_tsv(path.encode(), int(undirected), int(lt), int(renumber))
    try:
        n, m = R.ref_graph_nodes(g), R.ref_graph_edges(g)
        idx = np.zeros(n + 1, np.uint64)
        src = np.zeros(max(m, 1), np.uint32)
        w = np.zeros(max(m, 1), np.float32)
        rmap = np.zeros(max(n, 1), np.uint32)
        R.ref_graph_copy(g, _ptr(idx), _ptr(src), _ptr(w), _ptr(rmap))
        return n, idx, src[:m], w[:m], rmap[:n]
    finally:
        R.ref_graph_free(g)


def ref_sample(bin_path: str, model: str, count: int, seed: int = 0):
    R = reference()
    g = R.ref_graph_load(bin_path.encode())
    try:
        ne = ctypes.c_uint64()
        h = R.ref_sample(g, 0 if model == "IC" else 1, count, seed, ctypes.byref(ne))
        off = np.zeros(count + 1, dtype=np.uint64)
        vtx = np.zeros(max(ne.value, 1), dtype=np.uint32)
        R.ref_pool_copy(h, _ptr(off), _ptr(vtx))
        R.ref_pool_free(h)
        return off, vtx[: ne.value]
    finally:
        R.ref_graph_free(g)
