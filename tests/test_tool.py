"""The drop-in command-line tool ripples_b200/_lib/imm_b200: the reference
imm tool's options and JSON log, computing on the GPU."""
import json
import os
import subprocess

import numpy as np
import pytest

import ripples_b200 as rb
from conftest import GOLDEN, ROOT
from oracle import oracle as O

TOOL = os.path.join(ROOT, "ripples_b200", "_lib", "imm_b200")
KEYS = ["Algorithm", "Input", "Output", "DiffusionModel", "Epsilon", "K", "L", "NumThreads",
        "NumWalkWorkers", "NumCPUTeams", "NumGPUWalkWorkers", "PauseThreshold", "Total",
        "ThetaPrimeDeltas", "ThetaEstimation", "ThetaEstimationGenerateRRR",
        "ThetaEstimationMostInfluential", "Theta", "Counting", "Pivoting", "Microbenchmarking",
        "CPUBatchSize", "GPUBatchSize", "RRRSetSizeBytes", "GenerateRRRSets",
        "FindMostInfluentialSet", "Seeds"]


def run(*args):
    return subprocess.run([TOOL, *map(str, args)], capture_output=True, text=True, timeout=600)


def test_cli_rejects_bad_arguments():
    r = run("-i", "x.tsv", "-e", "0.5", "-d", "IC")
    assert r.returncode == 106 and "required" in r.stderr
    r = run("-i", "x.tsv", "-k", "3", "-e", "0.5", "-d", "IC", "--bogus")
    assert r.returncode == 106 and "unknown argument" in r.stderr
    r = run("-i", "x.tsv", "-k", "3", "-e", "0.5", "-d", "XX")
    assert r.returncode == 106
    r = run("-i", "x.tsv", "-k", "3", "-e", "0.5", "-d", "IC", "--scale-factor", "2")
    assert r.returncode == 106 and "scale factor" in r.stderr


@pytest.mark.gpu
def test_tool_tsv_matches_oracle(tmp_path):
    out = str(tmp_path / "log.json")
    r = run("-i", os.path.join(GOLDEN, "karate.tsv"), "-w", "-k", "4", "-e", "0.5", "-d", "IC",
            "-o", out)
    assert r.returncode == 0, r.stderr
    log = json.load(open(out))[0]
    assert all(k in log for k in KEYS)
    # the tool renumbers ids 1..34 -> 0..33 and reports input ids
    e = np.loadtxt(os.path.join(GOLDEN, "karate.tsv"))
    g = rb.HostGraph.from_edges(34, e[:, 0].astype(np.int64) - 1, e[:, 1].astype(np.int64) - 1,
                                e[:, 2].astype(np.float32))
    o = O.imm("IC", g.n, g.index, g.src, O.pack("IC", g.index, g.weights), 4, 0.5, seed=0)
    assert log["Seeds"] == [s + 1 for s in o["seeds"]]
    assert log["Theta"] == o["theta"] and log["ThetaPrimeDeltas"] == o["deltas"]


@pytest.mark.gpu
def test_tool_binary_matches_oracle(tmp_path):
    g = rb.HostGraph.rmat(12, 8 << 12, seed=41).with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=42)
    path = str(tmp_path / "g.bin")
    g.write_binary(path)
    out = str(tmp_path / "log.json")
    r = run("-i", path, "--reload-binary", "-k", "10", "-e", "0.5", "-d", "LT", "-o", out,
            "--seed", "3")
    assert r.returncode == 0, r.stderr
    log = json.load(open(out))[0]
    o = O.imm("LT", g.n, g.index, g.src, O.pack("LT", g.index, g.weights), 10, 0.5, seed=3)
    assert log["Seeds"] == o["seeds"] and log["Theta"] == o["theta"]
