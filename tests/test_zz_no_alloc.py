"""rip_sample_static: sampling for callers that cannot allocate device memory.

Some callers of this library cannot call cudaMalloc when they sample: a
serving process whose HBM is reserved up front by its own arena allocator, a
latency-critical loop where cudaMalloc/cudaFree would synchronise the device,
or a plugin host that forbids allocations outside its allocator.  For them
rip_sample_static takes the packed graph and the output buffers in their own
device memory and keeps its scratch in a fixed static device array.  This
test builds those buffers with torch (outside the call), runs two calls in a
row through the C ABI, and checks every set against what rip_sample -- the
allocating entry point -- produces for the same seed and set ids, and against
the CPU oracle: the sets must be identical, bit for bit.  A second case grows
sets past the 16 384-entry queues the array starts with, so the entry point
must re-run them with wider queues (fewer warps) and still return the same
sets.
"""
import ctypes

import numpy as np
import pytest

import ripples_b200 as rb
from oracle import oracle as O
from ripples_b200 import _lib

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def packed_graph(ctx, g, model):
    """The layout rip_graph_upload builds, in caller-owned device memory."""
    import torch
    dg = rb.DeviceGraph(ctx, g, model)
    thr = dg.thresholds()
    m = g.m
    m_pad = ((m + 3) & ~3) + 4
    rec = np.zeros((m_pad, 2), np.uint32)
    rec[:m, 0] = g.src
    rec[:m, 1] = thr
    d_edges = torch.from_numpy(rec.view(np.int32)).cuda()
    d_off = torch.from_numpy(g.index.astype(np.uint32).view(np.int32)).cuda()
    return dg, d_off, d_edges


def run_static(d_off, d_edges, g, model, seed, first, count, capacity):
    import torch
    d_vtx = torch.empty(capacity, dtype=torch.int32, device="cuda")
    d_so = torch.empty(count, dtype=torch.int64, device="cuda")
    d_sl = torch.empty(count, dtype=torch.int32, device="cuda")
    ne = ctypes.c_uint64()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = _lib.lib.rip_sample_static(_ptr(d_off), _ptr(d_edges), g.n, g.m,
                                    rb.MODEL_IC if model == "IC" else rb.MODEL_LT, seed,
                                    first, count, _ptr(d_vtx), capacity, _ptr(d_so),
                                    _ptr(d_sl), ctypes.byref(ne), stream)
    assert rc == 0, _lib.lib.rip_static_last_error().decode()
    vtx = d_vtx.cpu().numpy().view(np.uint32)
    so = d_so.cpu().numpy().view(np.uint64)
    sl = d_sl.cpu().numpy().view(np.uint32)
    assert int(ne.value) == int(sl.astype(np.uint64).sum())
    return [np.sort(vtx[int(so[i]):int(so[i]) + int(sl[i])]) for i in range(count)]


@pytest.mark.parametrize("model", ["IC", "LT"])
def test_static_sampling_matches_rip_sample(ctx, model):
    g = rb.HostGraph.rmat(12, 8 << 12, seed=21)
    g = g.with_weights(rb.WEIGHTS_UNIFORM, seed=22, lo=0.0, hi=0.3) if model == "IC" else \
        g.with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=22)
    seed, count = 77, 2500
    dg, d_off, d_edges = packed_graph(ctx, g, model)
    pool = rb.Pool(dg)
    pool.sample(count, seed=seed, sampler=rb.SAMPLER_PLAIN)
    pool.sample(count, seed=seed, sampler=rb.SAMPLER_PLAIN)
    off, vtx = pool.export()
    expected = [vtx[off[i]:off[i + 1]] for i in range(2 * count)]
    thr = O.pack(model, g.index, g.weights)
    ooff, ovtx, _ = O.sample(model, g.n, g.index, g.src, thr, seed, 0, 2 * count)
    capacity = int(off[-1]) + 1024
    # two calls in a row: sets [0, count) then [count, 2*count)
    for call in range(2):
        got = run_static(d_off, d_edges, g, model, seed, call * count, count, capacity)
        for i, s in enumerate(got):
            j = call * count + i
            assert np.array_equal(s, expected[j]), (call, i)
            assert np.array_equal(s, ovtx[ooff[j]:ooff[j + 1]]), (call, i)
    pool.close()
    dg.close()


def test_static_sampling_retries_sets_past_the_first_queues(ctx):
    # R-MAT 2^16 with p ~ U(0, 0.5): about two live in-edges per vertex, so
    # many sets hold a large share of the graph, more than the 16 384 entries
    # of the queues the scratch is first split into
    g = rb.HostGraph.rmat(16, 8 << 16, seed=5).with_weights(rb.WEIGHTS_UNIFORM, seed=6, lo=0.0,
                                                             hi=0.5)
    seed, count = 9, 200
    dg, d_off, d_edges = packed_graph(ctx, g, "IC")
    thr = O.pack("IC", g.index, g.weights)
    ooff, ovtx, _ = O.sample("IC", g.n, g.index, g.src, thr, seed, 0, count)
    for call in range(2):
        got = run_static(d_off, d_edges, g, "IC", seed, 0, count, count * g.n)
        assert max(len(x) for x in got) > (1 << 14)
        for i, x in enumerate(got):
            assert np.array_equal(x, ovtx[ooff[i]:ooff[i + 1]]), (call, i)
    dg.close()


def test_static_rejects_oversized_requests():
    import torch
    buf = torch.zeros(64, dtype=torch.int64, device="cuda")
    ne = ctypes.c_uint64()
    p = _ptr(buf)
    max_sets = 1 << 20  # RIP_STATIC_MAX_SETS
    rc = _lib.lib.rip_sample_static(p, p, 16, 0, rb.MODEL_IC, 0, 0, max_sets + 1, p, 64, p, p,
                                    ctypes.byref(ne), None)
    assert rc == -5
    assert b"at most" in _lib.lib.rip_static_last_error()
    # n too large for the static scratch
    rc = _lib.lib.rip_sample_static(p, p, 1 << 30, 0, rb.MODEL_IC, 0, 0, 1, p, 64, p, p,
                                    ctypes.byref(ne), None)
    assert rc == -5
    assert b"scratch" in _lib.lib.rip_static_last_error()
