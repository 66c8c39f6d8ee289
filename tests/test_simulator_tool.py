"""The drop-in simulator tool ripples_b200/_lib/simulator_b200: the reference
simulator's options, experiment file and JSON output, spreads on the GPU."""
import json
import os
import subprocess

import numpy as np
import pytest

import ripples_b200 as rb
from conftest import ROOT
from oracle import oracle as O

TOOL = os.path.join(ROOT, "ripples_b200", "_lib", "simulator_b200")


def run(*args):
    return subprocess.run([TOOL, *map(str, args)], capture_output=True, text=True, timeout=600)


def experiments(path, model, seeds, extra=None):
    rec = {"Algorithm": "IMM", "Input": "g", "DiffusionModel": model, "Epsilon": 0.5, "K":
           len(seeds), "Seeds": [int(s) for s in seeds]}
    rec.update(extra or {})
    with open(path, "w") as fh:
        json.dump([rec], fh)
    return str(path)


def test_cli_rejects_bad_input(tmp_path):
    g = tmp_path / "g.tsv"
    g.write_text("1 2\n2 3\n")
    e = experiments(tmp_path / "e.json", "IC", [1, 2])
    r = run("-i", g, "-e", e)
    assert r.returncode == 106 and "required" in r.stderr
    r = run("-i", g, "-e", e, "--replicas", "3", "--bogus")
    assert r.returncode == 106 and "unknown argument" in r.stderr
    bad = tmp_path / "bad.json"
    bad.write_text('[{"DiffusionModel": "IC", "Seeds": [1, 2}]')
    r = run("-i", g, "-e", bad, "--replicas", "3")
    assert r.returncode == 106 and "experiment file" in r.stderr
    r = run("-i", g, "-e", experiments(tmp_path / "x.json", "XX", [1]), "--replicas", "3")
    assert r.returncode == 106 and "DiffusionModel" in r.stderr
    r = run("-i", g, "-e", experiments(tmp_path / "y.json", "IC", [7]), "--replicas", "3")
    assert r.returncode == 106 and "seed 7" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("model,reload", [("IC", False), ("IC", True), ("LT", False)])
def test_tool_matches_oracle(tmp_path, model, reload):
    # every replica's [activated, levels] equals the oracle's forward
    # simulation on the graph the tool reads, seeds given in input ids
    g = rb.HostGraph.rmat(10, 8 << 10, seed=3)
    g = g.with_weights(rb.WEIGHTS_UNIFORM, seed=4, lo=0.0, hi=0.3) if model == "IC" else \
        g.with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=4)
    if reload:
        path = str(tmp_path / "gf.bin")
        g.write_binary(path, backward=False)
        args = ["--reload-binary"]
    else:
        src, dst = g.transpose_edges()
        path = str(tmp_path / "g.tsv")
        with open(path, "w") as fh:
            for s, d, w in zip(src, dst, g.weights):
                fh.write(f"{s}\t{d}\t{w:.9g}\n")
        args = ["-w", "--disable-renumbering"]
        g, _ = rb.HostGraph.read_tsv(path, weighted=True, renumber=False, model=model)
    seeds = [0, 5, 17, 100]
    e = experiments(tmp_path / "e.json", model, seeds, {"Extra": 1})
    out = str(tmp_path / "sim.json")
    r = run("-i", path, "-e", e, "--replicas", 300, "--seed", 9, "-o", out, *args)
    assert r.returncode == 0, r.stderr
    with open(out) as fh:
        rec = json.load(fh)[0]
    assert rec["DiffusionModel"] == model and rec["Seeds"] == seeds and rec["K"] == 4
    sims = np.asarray(rec["Simulations"], dtype=np.int64)
    if model == "IC":
        f = g.forward()
        thr = O.pack("IC", f.index, f.weights)
        _, sizes, levels = O.spread_ic(f.n, f.index, f.src, thr, seeds, 300, seed=9,
                                       with_levels=True)
    else:
        _, sizes, levels = O.spread_lt(g, seeds, 300, seed=9, with_levels=True)
    assert np.array_equal(sims[:, 0], sizes) and np.array_equal(sims[:, 1], levels)
