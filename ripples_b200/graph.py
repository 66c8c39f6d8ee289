"""Graphs on the host and on the device.

:class:`HostGraph` holds a backward CSR exactly as the reference's ``GraphBwd``
(include/ripples/graph.h:364-1086): ``index`` u64[n+1], ``src`` u32[m] (the
in-neighbours of v are ``src[index[v]:index[v+1]]``), ``weights`` f32[m].
Synthetic graphs (R-MAT, Erdos-Renyi) and weight models are produced by the
native library's host code, deterministically in their seeds.
:class:`Context`, :class:`DeviceGraph` and :class:`Pool` wrap the C ABI
objects ``rip_ctx``, ``rip_graph`` and ``rip_pool``.
"""
from __future__ import annotations

import ctypes
import weakref
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import RipError, check, lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


@dataclass
class HostGraph:
    n: int
    index: np.ndarray  # uint64[n+1]
    src: np.ndarray  # uint32[m]
    weights: Optional[np.ndarray] = None  # float32[m]

    @property
    def m(self) -> int:
        return int(self.src.shape[0])

    def in_degree(self) -> np.ndarray:
        return np.diff(self.index).astype(np.uint64)

    # ---- construction -------------------------------------------------
    @staticmethod
    def _from_native(n: int, pidx, psrc, m: int) -> "HostGraph":
        idx = np.ctypeslib.as_array(ctypes.cast(pidx, ctypes.POINTER(ctypes.c_uint64)),
                                    shape=(n + 1,)).copy()
        if m:
            src = np.ctypeslib.as_array(ctypes.cast(psrc, ctypes.POINTER(ctypes.c_uint32)),
                                        shape=(m,)).copy()
        else:
            src = np.zeros(0, dtype=np.uint32)
        lib.rip_free(pidx)
        lib.rip_free(psrc)
        return HostGraph(n, idx, src)

    @classmethod
    def rmat(cls, scale: int, num_edges: int, a: float = 0.57, b: float = 0.19,
             c: float = 0.19, seed: int = 0) -> "HostGraph":
        """Directed R-MAT graph on 2^scale vertices from ``num_edges`` draws
        (self-loops and duplicates removed)."""
        pidx, psrc, m = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_uint64()
        check(lib.rip_rmat_csr(scale, num_edges, a, b, c, seed, ctypes.byref(pidx),
                               ctypes.byref(psrc), ctypes.byref(m)), "rip_rmat_csr")
        return cls._from_native(1 << scale, pidx, psrc, m.value)

    @classmethod
    def erdos_renyi(cls, n: int, num_edges: int, seed: int = 0) -> "HostGraph":
        pidx, psrc, m = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_uint64()
        check(lib.rip_er_csr(n, num_edges, seed, ctypes.byref(pidx), ctypes.byref(psrc),
                             ctypes.byref(m)), "rip_er_csr")
        return cls._from_native(n, pidx, psrc, m.value)

    @classmethod
    def from_edges(cls, n: int, src: Sequence[int], dst: Sequence[int],
                   weights: Optional[Sequence[float]] = None) -> "HostGraph":
        """Backward CSR from a directed edge list (src -> dst); in-edges of
        each vertex ordered by source id.  Duplicates are kept."""
        s = np.asarray(src, dtype=np.uint64)
        d = np.asarray(dst, dtype=np.uint64)
        order = np.lexsort((s, d))
        s, d = s[order], d[order]
        idx = np.zeros(n + 1, dtype=np.uint64)
        np.add.at(idx, d.astype(np.int64) + 1, 1)
        idx = np.cumsum(idx).astype(np.uint64)
        w = None
        if weights is not None:
            w = np.asarray(weights, dtype=np.float32)[order]
        return cls(n, idx, s.astype(np.uint32), w)

    @staticmethod
    def _from_read(rc, n, m, pi, ps, pw, pm, where) -> Tuple["HostGraph", np.ndarray]:
        if rc != 0:
            raise RipError(rc, where, (lib.rip_read_error() or b"").decode())
        n, m = n.value, m.value

        def take(p, ctype, count, dtype):
            a = (np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctype)), shape=(count,)).copy()
                 if count else np.zeros(0, dtype=dtype))
            lib.rip_free(p)
            return a
        idx = take(pi, ctypes.c_uint64, n + 1, np.uint64)
        src = take(ps, ctypes.c_uint32, m, np.uint32)
        w = take(pw, ctypes.c_float, m, np.float32)
        rmap = take(pm, ctypes.c_uint32, n, np.uint32)
        return HostGraph(n, idx, src, w), rmap

    @classmethod
    def read_tsv(cls, path: str, weighted: bool = False, undirected: bool = False,
                 renumber: bool = True, model: str = "IC", distribution: str = "uniform",
                 mean: float = 0.5, variance: float = 1.0,
                 scale: float = 1.0) -> Tuple["HostGraph", np.ndarray]:
        """A TSV edge list read as the reference's loader and Graph constructor
        build its GraphBwd (``rip_read_tsv``); returns (graph, reverse id map)."""
        dist = {"uniform": _lib.DIST_UNIFORM, "normal": _lib.DIST_NORMAL,
                "const": _lib.DIST_CONST}.get(distribution, -1)
        o = _lib.TsvOptions(int(weighted), int(undirected), int(renumber), MODELS[model], dist,
                            mean, variance, scale)
        n, m = ctypes.c_uint32(), ctypes.c_uint64()
        pi, ps, pw, pm = (ctypes.c_void_p() for _ in range(4))
        rc = lib.rip_read_tsv(path.encode(), ctypes.byref(o), ctypes.byref(n), ctypes.byref(m),
                              ctypes.byref(pi), ctypes.byref(ps), ctypes.byref(pw),
                              ctypes.byref(pm))
        return cls._from_read(rc, n, m, pi, ps, pw, pm, "rip_read_tsv")

    @staticmethod
    def read_tsv_edges(path: str, weighted: bool = False, undirected: bool = False,
                       model: str = "IC", distribution: str = "uniform", mean: float = 0.5,
                       variance: float = 1.0,
                       scale: float = 1.0) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """A TSV file's edge list before any CSR is built (``rip_read_tsv_edges``):
        (src, dst, weights) in input ids, for ``DeviceGraph.from_edges``."""
        dist = {"uniform": _lib.DIST_UNIFORM, "normal": _lib.DIST_NORMAL,
                "const": _lib.DIST_CONST}.get(distribution, -1)
        o = _lib.TsvOptions(int(weighted), int(undirected), 1, MODELS[model], dist, mean,
                            variance, scale)
        m = ctypes.c_uint64()
        ps, pd, pw = (ctypes.c_void_p() for _ in range(3))
        rc = lib.rip_read_tsv_edges(path.encode(), ctypes.byref(o), ctypes.byref(m),
                                    ctypes.byref(ps), ctypes.byref(pd), ctypes.byref(pw))
        if rc != 0:
            raise RipError(rc, "rip_read_tsv_edges", (lib.rip_read_error() or b"").decode())
        mm = m.value
        try:
            src = np.ctypeslib.as_array(ctypes.cast(ps, ctypes.POINTER(ctypes.c_uint32)),
                                        shape=(max(mm, 1),))[:mm].copy()
            dst = np.ctypeslib.as_array(ctypes.cast(pd, ctypes.POINTER(ctypes.c_uint32)),
                                        shape=(max(mm, 1),))[:mm].copy()
            w = np.ctypeslib.as_array(ctypes.cast(pw, ctypes.POINTER(ctypes.c_float)),
                                      shape=(max(mm, 1),))[:mm].copy()
        finally:
            for x in (ps, pd, pw):
                lib.rip_free(x)
        return src, dst, w

    @classmethod
    def read_binary(cls, path: str, scale: float = 1.0,
                    forward: bool = False) -> Tuple["HostGraph", np.ndarray]:
        """The reference binary format (``rip_read_binary``; with ``forward``
        the forward direction, ``rip_read_binary_forward``, whose CSR is indexed
        by source); returns (graph, reverse id map)."""
        n, m = ctypes.c_uint32(), ctypes.c_uint64()
        pi, ps, pw, pm = (ctypes.c_void_p() for _ in range(4))
        fn = lib.rip_read_binary_forward if forward else lib.rip_read_binary
        rc = fn(path.encode(), scale, ctypes.byref(n), ctypes.byref(m), ctypes.byref(pi),
                ctypes.byref(ps), ctypes.byref(pw), ctypes.byref(pm))
        return cls._from_read(rc, n, m, pi, ps, pw, pm, "rip_read_binary")

    def transposed(self) -> "HostGraph":
        """The CSR of the transposed graph (``rip_transpose_csr``): in-lists
        become out-lists, each ordered by the other endpoint."""
        pi, pa, pw = (ctypes.c_void_p() for _ in range(3))
        idx = np.ascontiguousarray(self.index, dtype=np.uint64)
        adj = np.ascontiguousarray(self.src, dtype=np.uint32)
        w = np.ascontiguousarray(self.weights if self.weights is not None
                                 else np.zeros(self.m, np.float32), dtype=np.float32)
        rc = lib.rip_transpose_csr(self.n, self.m, _ptr(idx), _ptr(adj), _ptr(w),
                                   ctypes.byref(pi), ctypes.byref(pa), ctypes.byref(pw))
        if rc != 0:
            raise RipError(rc, "rip_transpose_csr", (lib.rip_read_error() or b"").decode())

        def take(p, ctype, count, dtype):
            a = (np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctype)), shape=(count,)).copy()
                 if count else np.zeros(0, dtype=dtype))
            lib.rip_free(p)
            return a
        return HostGraph(self.n, take(pi, ctypes.c_uint64, self.n + 1, np.uint64),
                         take(pa, ctypes.c_uint32, self.m, np.uint32),
                         take(pw, ctypes.c_float, self.m, np.float32))

    def with_weights(self, kind: int, seed: int = 1, lo: float = 0.0,
                     hi: float = 1.0) -> "HostGraph":
        w = np.empty(self.m, dtype=np.float32)
        check(lib.rip_make_weights(kind, self.n, _ptr(self.index), self.m, seed, lo, hi,
                                   _ptr(w)), "rip_make_weights")
        return HostGraph(self.n, self.index, self.src, w)

    def write_binary(self, path: str, backward: bool = True) -> None:
        """Writes the reference binary format (include/ripples/graph.h:700-771)."""
        assert self.weights is not None
        check(lib.rip_write_binary(path.encode(), self.n, self.m, _ptr(self.index),
                                   _ptr(self.src), _ptr(self.weights), 1 if backward else 0),
              "rip_write_binary")

    def forward(self) -> "HostGraph":
        """The forward CSR of the same graph in this class's layout: ``index``
        over source vertices, ``src`` holding each out-edge's target (ordered
        by target id), ``weights`` p(u -> v) -- what ``rip_spread_ic`` takes."""
        s, d = self.transpose_edges()
        return HostGraph.from_edges(self.n, d, s, self.weights)

    def transpose_edges(self) -> Tuple[np.ndarray, np.ndarray]:
        """(src, dst) arrays of the directed edges, in backward-CSR order."""
        dst = np.repeat(np.arange(self.n, dtype=np.uint32), np.diff(self.index).astype(np.int64))
        return self.src.copy(), dst


class Context:
    """One CUDA device + stream (``rip_ctx``).  The context owns the graphs
    and pools created on it: closing it frees them, and their Python handles
    become inert."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        h = ctypes.c_void_p()
        check(lib.rip_ctx_create(device, hbm_budget, ctypes.byref(h)), "rip_ctx_create")
        self.h = h
        self.device = device
        self._children = weakref.WeakSet()

    def close(self) -> None:
        if self.h:
            for ch in list(self._children):
                ch._invalidate()
            lib.rip_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self) -> None:
        check(lib.rip_sync(self.h), "rip_sync", self.h)

    def coin_rate(self) -> float:
        """Measured coins per second of the IC coin function alone
        (``rip_coin_rate``): the ceiling of the samplers on uniform-threshold
        graphs."""
        r = ctypes.c_double()
        check(lib.rip_coin_rate(self.h, ctypes.byref(r)), "rip_coin_rate", self.h)
        return r.value

    def memory(self) -> Tuple[int, int]:
        used, budget = ctypes.c_size_t(), ctypes.c_size_t()
        check(lib.rip_ctx_memory(self.h, ctypes.byref(used), ctypes.byref(budget)),
              "rip_ctx_memory", self.h)
        return used.value, budget.value


MODELS = {"IC": _lib.MODEL_IC, "LT": _lib.MODEL_LT}


class DeviceGraph:
    """A packed backward CSR resident in HBM (``rip_graph``)."""

    def __init__(self, ctx: Context, g: HostGraph, model: str):
        assert g.weights is not None, "weights required"
        self.ctx, self.model, self.n, self.m = ctx, model, g.n, g.m
        h = ctypes.c_void_p()
        idx = np.ascontiguousarray(g.index, dtype=np.uint64)
        src = np.ascontiguousarray(g.src, dtype=np.uint32)
        w = np.ascontiguousarray(g.weights, dtype=np.float32)
        check(lib.rip_graph_upload(ctx.h, _ptr(idx), _ptr(src), _ptr(w), g.n, g.m,
                                   MODELS[model], ctypes.byref(h)), "rip_graph_upload", ctx.h)
        self.h = h
        self._pools = weakref.WeakSet()
        ctx._children.add(self)

    def _invalidate(self) -> None:
        for p in list(self._pools):
            p._invalidate()
        self.h = None

    @classmethod
    def rmat_on_device(cls, ctx: Context, scale: int, num_edges: int, model: str,
                       weights: int, seed: int = 0, weight_seed: int = 1, lo: float = 0.0,
                       hi: float = 1.0, a: float = 0.57, b: float = 0.19,
                       c: float = 0.19) -> "DeviceGraph":
        """The graph HostGraph.rmat(...).with_weights(...) would build, built on
        the device: R-MAT keys by the library, sort + unique by torch (input
        plumbing), CSR + weights + packing by the library."""
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        keys = torch.empty(num_edges, dtype=torch.int64, device=dev)
        check(lib.rip_rmat_keys_device(ctx.h, scale, 0, num_edges, a, b, c, seed,
                                       ctypes.c_void_p(keys.data_ptr())),
              "rip_rmat_keys_device", ctx.h)
        return cls._from_keys(ctx, keys, 1 << scale, model, weights, weight_seed, lo, hi)

    @classmethod
    def erdos_renyi_on_device(cls, ctx: Context, n: int, num_edges: int, model: str,
                              weights: int, seed: int = 0, weight_seed: int = 1,
                              lo: float = 0.0, hi: float = 1.0) -> "DeviceGraph":
        """HostGraph.erdos_renyi(...).with_weights(...), built on the device."""
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        keys = torch.empty(num_edges, dtype=torch.int64, device=dev)
        check(lib.rip_er_keys_device(ctx.h, n, 0, num_edges, seed,
                                     ctypes.c_void_p(keys.data_ptr())),
              "rip_er_keys_device", ctx.h)
        return cls._from_keys(ctx, keys, n, model, weights, weight_seed, lo, hi)

    @classmethod
    def _from_keys(cls, ctx, keys, n, model, weights, weight_seed, lo, hi) -> "DeviceGraph":
        import torch
        keys = torch.unique(keys[keys >= 0])  # drop self-loops (~0), sort, dedup
        torch.cuda.synchronize(keys.device)
        h = ctypes.c_void_p()
        check(lib.rip_graph_from_keys(ctx.h, ctypes.c_void_p(keys.data_ptr()), keys.numel(),
                                      n, weights, weight_seed, lo, hi, MODELS[model],
                                      ctypes.byref(h)), "rip_graph_from_keys", ctx.h)
        m = keys.numel()
        del keys
        obj = cls.__new__(cls)
        obj.ctx, obj.model, obj.n, obj.m, obj.h = ctx, model, n, m, h
        obj._pools = weakref.WeakSet()
        ctx._children.add(obj)
        return obj

    def uniform_thresholds(self, enable: Optional[bool] = None) -> bool:
        """Whether the per-vertex uniform IC thresholds exist
        (``rip_graph_uniform_thresholds``); ``enable`` turns their use on or
        off (sets never depend on it)."""
        avail = ctypes.c_int()
        check(lib.rip_graph_uniform_thresholds(self.h, -1 if enable is None else int(enable),
                                               ctypes.byref(avail)),
              "rip_graph_uniform_thresholds", self.ctx.h)
        return bool(avail.value)

    @classmethod
    def from_edges(cls, ctx: "Context", src, dst, weights, model: str,
                   renumber: bool = True) -> "DeviceGraph":
        """The graph built on the device from a host edge list
        (``rip_graph_from_edges``): renumbering, transpose and packing on the
        GPU.  ``id_map()`` gives internal id -> input id."""
        self = cls.__new__(cls)
        s = np.ascontiguousarray(src, dtype=np.uint32)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        w = np.ascontiguousarray(weights, dtype=np.float32)
        h = ctypes.c_void_p()
        check(lib.rip_graph_from_edges(ctx.h, _ptr(s), _ptr(d), _ptr(w), len(s),
                                       int(renumber), MODELS[model], ctypes.byref(h)),
              "rip_graph_from_edges", ctx.h)
        n, m = ctypes.c_uint32(), ctypes.c_uint64()
        check(lib.rip_graph_info(h, ctypes.byref(n), ctypes.byref(m), None), "rip_graph_info",
              ctx.h)
        self.ctx, self.model, self.n, self.m, self.h = ctx, model, n.value, m.value, h
        self._pools = weakref.WeakSet()
        ctx._children.add(self)
        return self

    def id_map(self) -> np.ndarray:
        out = np.zeros(max(self.n, 1), dtype=np.uint32)
        check(lib.rip_graph_id_map(self.h, _ptr(out)), "rip_graph_id_map", self.ctx.h)
        return out[: self.n]

    @property
    def branching(self) -> float:
        """Branching factor of a reverse BFS (IC; ``rip_graph_branching``)."""
        b = ctypes.c_double()
        check(lib.rip_graph_branching(self.h, ctypes.byref(b)), "rip_graph_branching",
              self.ctx.h)
        return b.value

    def export(self) -> Tuple[np.ndarray, np.ndarray]:
        idx = np.zeros(self.n + 1, dtype=np.uint64)
        src = np.zeros(max(self.m, 1), dtype=np.uint32)
        check(lib.rip_graph_export(self.h, _ptr(idx), _ptr(src)), "rip_graph_export",
              self.ctx.h)
        return idx, src[: self.m]

    TUNE_NAMES = ("plain, heavy>2^18 grid BFS", "plain, heavy>2^14 grid BFS",
                  "plain, heavy>2^18 CTA per set, 1024-thread CTAs", "fused 64", "fused 128",
                  "fused 256", "plain 40 warps/SM, heavy>2^18 grid BFS",
                  "plain 40 warps/SM, heavy>2^18 CTA per set, 256-thread CTAs",
                  "plain, heavy>2^18 CTA per set, 256-thread CTAs",
                  "plain, heavy>2^16 CTA per set, 256-thread CTAs")

    def autotune(self, seed: int = 0, pilot: int = 0) -> dict:
        """Times each IC sampler configuration on a pilot of sets and keeps the
        fastest for this graph (``rip_graph_autotune``)."""
        ms = np.zeros(len(self.TUNE_NAMES), dtype=np.float64)
        ch = ctypes.c_int()
        check(lib.rip_graph_autotune(self.h, seed, pilot, _ptr(ms), ctypes.byref(ch)),
              "rip_graph_autotune", self.ctx.h)
        return {"choice": ch.value, "name": self.TUNE_NAMES[ch.value],
                "ms": {n: float(t) for n, t in zip(self.TUNE_NAMES, ms) if t >= 0}}

    def thresholds(self) -> np.ndarray:
        out = np.empty(self.m, dtype=np.uint32)
        check(lib.rip_graph_thresholds(self.h, _ptr(out)), "rip_graph_thresholds", self.ctx.h)
        return out

    def close(self) -> None:
        if self.h:
            for p in list(self._pools):
                p._invalidate()  # freed by rip_graph_destroy
            if self.ctx.h:
                lib.rip_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Pool:
    """Device-resident flat RRR pool (``rip_pool``)."""

    def __init__(self, graph: DeviceGraph):
        self.graph, self.ctx = graph, graph.ctx
        h = ctypes.c_void_p()
        check(lib.rip_pool_create(self.ctx.h, graph.h, ctypes.byref(h)), "rip_pool_create",
              self.ctx.h)
        self.h = h
        graph._pools.add(self)
        self.ctx._children.add(self)

    def _invalidate(self) -> None:
        self.h = None

    def close(self) -> None:
        if self.h:
            if self.ctx.h and self.graph.h:
                lib.rip_pool_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc, where):
        check(rc, where, self.ctx.h)

    def configure(self, colors: int = 64, slots: int = 0, log_capacity: int = 0) -> None:
        self._chk(lib.rip_pool_configure(self.h, colors, slots, log_capacity),
                  "rip_pool_configure")

    def plain_occupancy(self, blocks_per_sm: int) -> None:
        """One-set-per-warp IC kernel variant: 0 (no register cap) or 5."""
        self._chk(lib.rip_pool_plain_occupancy(self.h, blocks_per_sm),
                  "rip_pool_plain_occupancy")

    def heavy_batch(self, min_sets: int) -> None:
        """Heavy IC sets pending from which the grid-wide multi-colour BFS
        grows them (0 = one CTA per set)."""
        self._chk(lib.rip_pool_heavy_batch(self.h, min_sets), "rip_pool_heavy_batch")

    def heavy_block(self, threads: int) -> None:
        """Block shape (128/256/512/1024 threads) of the CTA-per-set kernel
        for heavy IC sets."""
        self._chk(lib.rip_pool_heavy_block(self.h, threads), "rip_pool_heavy_block")

    def select_guess(self, percent: int) -> None:
        """First-fetch threshold of reference-heap picks, % of the previous
        gain (0 = adaptive)."""
        self._chk(lib.rip_pool_select_guess(self.h, percent), "rip_pool_select_guess")

    def work_caps(self, plain: int, fused: int) -> None:
        self._chk(lib.rip_pool_work_caps(self.h, plain, fused), "rip_pool_work_caps")

    def clear(self) -> None:
        self._chk(lib.rip_pool_clear(self.h), "rip_pool_clear")

    @property
    def num_sets(self) -> int:
        s, e = ctypes.c_uint64(), ctypes.c_uint64()
        self._chk(lib.rip_pool_info(self.h, ctypes.byref(s), ctypes.byref(e)), "rip_pool_info")
        return s.value

    @property
    def num_elements(self) -> int:
        s, e = ctypes.c_uint64(), ctypes.c_uint64()
        self._chk(lib.rip_pool_info(self.h, ctypes.byref(s), ctypes.byref(e)), "rip_pool_info")
        return e.value

    def sample(self, count: int, seed: int = 0, sampler: int = _lib.SAMPLER_AUTO) -> None:
        self._chk(lib.rip_sample(self.h, seed, count, sampler), "rip_sample")

    def skip(self, count: int) -> None:
        """Appends ``count`` empty sets (ids another shard samples;
        ``rip_pool_skip``)."""
        self._chk(lib.rip_pool_skip(self.h, count), "rip_pool_skip")

    def shard_begin(self, num_sets: int, d_sum: int) -> int:
        """This pool's counts over sets [0, num_sets) into the device array
        at address ``d_sum`` (n uint32), and its vertex -> sets index
        (``rip_shard_begin``); returns those sets' element count."""
        e = ctypes.c_uint64()
        self._chk(lib.rip_shard_begin(self.h, num_sets, d_sum, ctypes.byref(e)),
                  "rip_shard_begin")
        return e.value

    def shard_pick(self, d_sum: int) -> Tuple[int, int]:
        """(vertex, count) of the largest entry of the device array at
        ``d_sum``, lowest id on ties (``rip_shard_pick``)."""
        v, g = ctypes.c_uint32(), ctypes.c_uint64()
        self._chk(lib.rip_shard_pick(self.h, d_sum, ctypes.byref(v), ctypes.byref(g)),
                  "rip_shard_pick")
        return v.value, g.value

    def shard_cover(self, vertex: int, gain: int, d_sum: int) -> None:
        """Covers this pool's sets holding ``vertex`` and writes its updated
        counts to ``d_sum`` (``rip_shard_cover``)."""
        self._chk(lib.rip_shard_cover(self.h, vertex, gain, d_sum), "rip_shard_cover")

    def shard_cover_list(self, vertex: int, gain: int, d_dec: int, capacity: int) -> int:
        """Covers this pool's sets holding ``vertex`` and writes their members
        to the device array at ``d_dec``; returns how many
        (``rip_shard_cover_list``)."""
        c = ctypes.c_uint64()
        self._chk(lib.rip_shard_cover_list(self.h, vertex, gain, d_dec, capacity,
                                           ctypes.byref(c)), "rip_shard_cover_list")
        return c.value

    def shard_apply(self, d_sum: int, d_dec: int, count: int) -> None:
        """Subtracts one from ``d_sum`` per listed vertex (``rip_shard_apply``)."""
        self._chk(lib.rip_shard_apply(self.h, d_sum, d_dec, count), "rip_shard_apply")

    def export(self, first: int = 0, count: Optional[int] = None) -> Tuple[np.ndarray, np.ndarray]:
        if count is None:
            count = self.num_sets - first
        off = np.zeros(count + 1, dtype=np.uint64)
        self._chk(lib.rip_pool_export(self.h, first, count, _ptr(off), None), "rip_pool_export")
        vtx = np.zeros(max(int(off[-1]), 1), dtype=np.uint32)
        self._chk(lib.rip_pool_export(self.h, first, count, _ptr(off), _ptr(vtx)),
                  "rip_pool_export")
        return off, vtx[: int(off[-1])]

    def import_sets(self, offsets: np.ndarray, vertices: np.ndarray) -> None:
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        vtx = np.ascontiguousarray(vertices, dtype=np.uint32)
        if vtx.size == 0:
            vtx = np.zeros(1, dtype=np.uint32)
        self._chk(lib.rip_pool_import(self.h, _ptr(off), _ptr(vtx), len(off) - 1),
                  "rip_pool_import")

    def stats(self) -> np.ndarray:
        st = np.zeros(8, dtype=np.uint64)
        self._chk(lib.rip_pool_stats(self.h, _ptr(st)), "rip_pool_stats")
        return st

    def timing(self) -> Tuple[float, int, float]:
        ms, n, sms = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_double()
        self._chk(lib.rip_pool_timing(self.h, ctypes.byref(ms), ctypes.byref(n),
                                      ctypes.byref(sms)), "rip_pool_timing")
        return ms.value, n.value, sms.value

    def select_profile(self) -> dict:
        out = np.zeros(12, dtype=np.float64)
        self._chk(lib.rip_select_profile(self.h, _ptr(out)), "rip_select_profile")
        keys = ["prep_ms", "heap_ms", "picks_ms", "pops", "seeds", "candidates", "selections",
                "cover_fetch_ms", "full_fetches", "pop_ms", "collect_ms", "fetch_rounds"]
        return dict(zip(keys, out.tolist()))

    def count(self, num_sets: Optional[int] = None) -> np.ndarray:
        if num_sets is None:
            num_sets = self.num_sets
        out = np.zeros(self.graph.n, dtype=np.uint32)
        self._chk(lib.rip_count(self.h, num_sets, _ptr(out)), "rip_count")
        return out

    def select(self, k: int, num_sets: Optional[int] = None,
               tiebreak: int = _lib.TIE_REF_HEAP):
        """Greedy max coverage; returns (f, seeds, gains)."""
        if num_sets is None:
            num_sets = self.num_sets
        seeds = np.zeros(max(k, 1), dtype=np.uint32)
        gains = np.zeros(max(k, 1), dtype=np.uint64)
        ns, f = ctypes.c_uint32(), ctypes.c_double()
        self._chk(lib.rip_select(self.h, num_sets, k, tiebreak, _ptr(seeds), _ptr(gains),
                                 ctypes.byref(ns), ctypes.byref(f)), "rip_select")
        return f.value, seeds[: ns.value].copy(), gains[: ns.value].copy()

    def select_counts(self) -> np.ndarray:
        out = np.zeros(self.graph.n, dtype=np.uint32)
        self._chk(lib.rip_select_counts(self.h, _ptr(out)), "rip_select_counts")
        return out

    def coverage(self, seeds, num_sets: Optional[int] = None) -> int:
        """Sets among the first ``num_sets`` holding at least one of ``seeds``
        (``rip_coverage``, OPIM-C's FindCoverage)."""
        sd = np.ascontiguousarray(seeds, dtype=np.uint32)
        out = ctypes.c_uint64()
        self._chk(lib.rip_coverage(self.h, self.num_sets if num_sets is None else num_sets,
                                   _ptr(sd) if sd.size else None, int(sd.size),
                                   ctypes.byref(out)), "rip_coverage")
        return out.value

    def imm(self, k: int, epsilon: float, l: float = 1.0, seed: int = 0,
            tiebreak: int = _lib.TIE_REF_HEAP, sampler: int = _lib.SAMPLER_AUTO):
        seeds = np.zeros(max(k, 1), dtype=np.uint32)
        ns = ctypes.c_uint32()
        rec = _lib.ImmRecord()
        self._chk(lib.rip_imm_pool(self.h, k, epsilon, l, seed, tiebreak, sampler,
                                   _ptr(seeds), ctypes.byref(ns), ctypes.byref(rec)),
                  "rip_imm_pool")
        return seeds[: ns.value].copy(), rec


def sample_multi(ctx: Context, pools, seeds, counts) -> None:
    """Extends every pool by counts[i] sets of seeds[i] in one launch
    (``rip_sample_multi``); the sets equal what ``Pool.sample`` would add."""
    n = len(pools)
    hp = (ctypes.c_void_p * n)(*[p.h.value if hasattr(p.h, "value") else p.h for p in pools])
    sd = np.ascontiguousarray(seeds, dtype=np.uint64)
    ct = np.ascontiguousarray(counts, dtype=np.uint64)
    check(lib.rip_sample_multi(ctx.h, hp, _ptr(sd), _ptr(ct), n), "rip_sample_multi", ctx.h)


def spread_ic(graph: DeviceGraph, seeds, replicas: int, seed: int = 0,
              with_sizes: bool = False, with_levels: bool = False):
    """Forward Monte Carlo spread of ``seeds`` under IC (``rip_spread_ic``):
    ``graph`` is an IC ``DeviceGraph`` of the FORWARD CSR
    (``HostGraph.forward()``).  Returns the mean reached count, and with
    ``with_sizes`` / ``with_levels`` also each replica's count / BFS levels."""
    sd = np.ascontiguousarray(seeds, dtype=np.uint32)
    sizes = np.zeros(max(replicas, 1), dtype=np.uint32) if with_sizes else None
    levels = np.zeros(max(replicas, 1), dtype=np.uint32) if with_levels else None
    out = ctypes.c_double()
    check(lib.rip_spread_ic(graph.h, _ptr(sd) if sd.size else None, int(sd.size), replicas, seed,
                            _ptr(sizes), _ptr(levels), ctypes.byref(out)), "rip_spread_ic",
          graph.ctx.h)
    return _spread_result(out.value, sizes, levels, replicas)


def _spread_result(mean, sizes, levels, replicas):
    res = [mean]
    if sizes is not None:
        res.append(sizes[:replicas])
    if levels is not None:
        res.append(levels[:replicas])
    return res[0] if len(res) == 1 else tuple(res)


def opimc(r1: Pool, r2: Pool, k: int, epsilon: float, delta: float, seed: int = 0,
          tiebreak: int = _lib.TIE_REF_HEAP, sampler: int = _lib.SAMPLER_AUTO):
    """OPIM-C on two pools of one graph (``rip_opimc_pool``): (seeds, record)."""
    seeds = np.zeros(max(k, 1), dtype=np.uint32)
    ns = ctypes.c_uint32()
    rec = _lib.OpimcRecord()
    check(lib.rip_opimc_pool(r1.h, r2.h, k, epsilon, delta, seed, tiebreak, sampler,
                             _ptr(seeds), ctypes.byref(ns), ctypes.byref(rec)),
          "rip_opimc_pool", r1.graph.ctx.h)
    return seeds[: ns.value].copy(), rec


def spread_lt(forward: DeviceGraph, backward: DeviceGraph, seeds, replicas: int,
              seed: int = 0, with_sizes: bool = False, with_levels: bool = False):
    """Forward Monte Carlo spread of ``seeds`` under LT (``rip_spread_lt``):
    ``forward`` holds the forward CSR (``HostGraph.forward()``, any model),
    ``backward`` is the same graph's LT ``DeviceGraph``.  Returns the mean
    reached count, and with ``with_sizes`` also each replica's count."""
    sd = np.ascontiguousarray(seeds, dtype=np.uint32)
    sizes = np.zeros(max(replicas, 1), dtype=np.uint32) if with_sizes else None
    levels = np.zeros(max(replicas, 1), dtype=np.uint32) if with_levels else None
    out = ctypes.c_double()
    check(lib.rip_spread_lt(forward.h, backward.h, _ptr(sd) if sd.size else None, int(sd.size),
                            replicas, seed, _ptr(sizes), _ptr(levels), ctypes.byref(out)),
          "rip_spread_lt", forward.ctx.h)
    return _spread_result(out.value, sizes, levels, replicas)


class Query:
    """One IMM query (``rip_imm_query``) with its seed buffer."""

    def __init__(self, graph: DeviceGraph, k: int, epsilon: float, l: float = 1.0,
                 seed: int = 0, tiebreak: int = _lib.TIE_LOWEST_ID):
        self.graph = graph
        self.buf = np.zeros(max(k, 1), dtype=np.uint32)
        self.q = _lib.ImmQuery()
        self.q.graph = graph.h.value if hasattr(graph.h, "value") else graph.h
        self.q.k, self.q.epsilon, self.q.l = k, epsilon, l
        self.q.seed, self.q.tiebreak = seed, tiebreak
        self.q.seeds = self.buf.ctypes.data
        self.submitted_at = None

    @property
    def done(self) -> bool:
        return bool(self.q.done)

    @property
    def status(self) -> int:
        return self.q.status

    @property
    def seeds(self) -> np.ndarray:
        return self.buf[: self.q.num_seeds].copy()

    @property
    def record(self):
        return self.q.record

    @property
    def latency_ms(self) -> float:
        return self.q.latency_ms


def imm_batch(ctx: Context, queries) -> None:
    """Runs the queries to completion as one continuous batch (``rip_imm_batch``)."""
    n = len(queries)
    arr = (_lib.ImmQuery * n)()
    for i, q in enumerate(queries):
        arr[i] = q.q
    check(lib.rip_imm_batch(ctx.h, arr, n), "rip_imm_batch", ctx.h)
    for i, q in enumerate(queries):
        q.q = arr[i]


class Server:
    """Request loop over resident pools (``rip_server``): ``submit`` queues a
    query, ``tick`` admits what fits and advances every admitted query by one
    round."""

    def __init__(self, ctx: Context, footprint_budget: int = 0, max_active: int = 16):
        h = ctypes.c_void_p()
        check(lib.rip_server_create(ctx.h, footprint_budget, max_active, ctypes.byref(h)),
              "rip_server_create", ctx.h)
        self.ctx, self.h = ctx, h
        self._live = []
        ctx._children.add(self)

    def _invalidate(self) -> None:
        self.h = None  # freed with its context

    def submit(self, q: Query) -> Query:
        check(lib.rip_server_submit(self.h, ctypes.byref(q.q)), "rip_server_submit", self.ctx.h)
        self._live.append(q)
        return q

    def tick(self) -> int:
        done = ctypes.c_uint32()
        check(lib.rip_server_tick(self.h, ctypes.byref(done)), "rip_server_tick", self.ctx.h)
        self._live = [q for q in self._live if not q.q.done]
        return done.value

    def pending(self) -> Tuple[int, int]:
        a, qd = ctypes.c_uint32(), ctypes.c_uint32()
        check(lib.rip_server_pending(self.h, ctypes.byref(a), ctypes.byref(qd)),
              "rip_server_pending", self.ctx.h)
        return a.value, qd.value

    def stats(self) -> dict:
        out = np.zeros(10, dtype=np.uint64)
        check(lib.rip_server_stats(self.h, _ptr(out)), "rip_server_stats", self.ctx.h)
        keys = ("ticks", "completed", "graph_launches", "pools", "admitted_bytes", "tick_us",
                "suspended", "sample_us", "index_us", "index_select_us")
        return {k: int(v) for k, v in zip(keys, out)}

    def drain(self) -> None:
        while any(self.pending()):
            self.tick()

    def close(self) -> None:
        if self.h and self.ctx.h:
            lib.rip_server_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
