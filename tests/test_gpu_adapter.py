"""The drop-in C++ adapter (include/ripples_b200/imm_adapter.hpp), compiled
against the reference's own headers (oracle/_ref/adapter_imm), drives
ripples::IMM / GenerateRRRSets / FindMostInfluentialSet on the GPU and gives
the oracle's results."""
import json
import os
import subprocess

import numpy as np
import pytest

import ripples_b200 as rb
from conftest import ROOT
from oracle import oracle as O

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "oracle", "_ref", "adapter_imm")


@pytest.mark.parametrize("model", ["IC", "LT"])
def test_adapter_through_reference_api(tmp_path, model):
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/adapter_imm not built")
    g = rb.HostGraph.rmat(12, 8 << 12, seed=31)
    g = g.with_weights(rb.WEIGHTS_UNIFORM, seed=32, lo=0.0, hi=0.2) if model == "IC" else \
        g.with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=32)
    path = str(tmp_path / "g.bin")
    g.write_binary(path, backward=True)
    k, eps, seed, nsets = 10, 0.5, 5, 3000
    out = subprocess.run([EXE, path, model, str(k), str(eps), str(seed), str(nsets)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    r = json.loads(out.stdout)
    thr = O.pack(model, g.index, g.weights)
    o = O.imm(model, g.n, g.index, g.src, thr, k, eps, seed=seed)
    assert r["imm_seeds"] == o["seeds"] and r["theta"] == o["theta"]
    assert r["deltas"] == o["deltas"]
    off, vtx, _ = O.sample(model, g.n, g.index, g.src, thr, seed, 0, nsets)
    assert r["sets"] == nsets and r["elements"] == len(vtx) and r["sorted"]
    f, seeds, _, _ = O.select(g.n, off, vtx, k, 0)
    assert r["select_seeds"] == seeds.tolist() and r["f"] == f
    half = nsets // 2
    f2, seeds2, _, _ = O.select(g.n, off[:half + 1], vtx[:int(off[half])], k, 0)
    assert r["half_seeds"] == seeds2.tolist() and r["half_f"] == f2
    # the record: one walk iteration (one GPU walk) for the one GenerateRRRSets
    # call, one Counting and one Pivoting entry per FindMostInfluentialSet
    assert r["walk_iterations"] == 1 and r["walk_sets"] == nsets and r["gpu_walks"] == 1
    assert r["counting"] == 2 and r["pivoting"] == 2
