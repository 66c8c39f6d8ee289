"""North-star check 4: the spread of our IMM seeds, measured with the
reference's own Monte Carlo simulator (include/ripples/diffusion_simulation.h,
driven like tools/simulator.cc), is within 1% of the spread of the seeds the
reference's imm tool picks on the same graph.

Our seeds come from the oracle's IMM, which the GPU tests prove bit-identical
to the device IMM (same sets, same selection), so this runs on the CPU."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

import ripples_b200 as rb
from oracle import oracle as O
from conftest import ROOT

IMM_EXE = os.path.join(ROOT, "oracle", "_ref", "imm")


def reference_seeds(path, model, k, eps, parallel):
    out = tempfile.mktemp(suffix=".json")
    cmd = [IMM_EXE, "-i", path, "--reload-binary", "-d", model, "-k", str(k), "-e", str(eps),
           "-o", out] + (["-p"] if parallel else [])
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                   env=dict(os.environ, OMP_NUM_THREADS="4"), timeout=600)
    with open(out) as fh:
        rec = json.load(fh)[0]
    os.unlink(out)
    return rec["Seeds"]


@pytest.mark.parametrize("model,scale,draws,k,eps,reps", [
    ("IC", 14, 1 << 18, 20, 0.5, 3000),  # the 2^14-vertex IC configuration
    ("LT", 12, 8 << 12, 20, 0.5, 400),   # a reduced LT configuration
])
def test_spread_within_one_percent_of_reference(tmp_path, model, scale, draws, k, eps, reps):
    # Replicas: the standard error of the mean spread is below 0.1% of the
    # spread at these counts, well inside the 1% bound.
    R = O.reference()
    if R is None or not os.path.exists(IMM_EXE):
        pytest.skip("oracle/_ref not built")
    g = rb.HostGraph.rmat(scale, draws, seed=0)
    g = g.with_weights(rb.WEIGHTS_UNIFORM, seed=1, lo=0.0, hi=0.1) if model == "IC" else \
        g.with_weights(rb.WEIGHTS_LT_NORMALIZED, seed=1)
    bwd = str(tmp_path / "g.bin")
    fwd = str(tmp_path / "gf.bin")
    g.write_binary(bwd, backward=True)
    g.write_binary(fwd, backward=False)
    ref = reference_seeds(bwd, model, k, eps, parallel=(model == "IC"))
    thr = O.pack(model, g.index, g.weights)
    ours = O.imm(model, g.n, g.index, g.src, thr, k, eps, seed=0)["seeds"]
    assert len(ours) == len(ref) == k
    m = 0 if model == "IC" else 1
    s_ref = R.ref_simulate(fwd.encode(), m, np.asarray(ref, np.uint32).ctypes.data, k, reps, 0)
    s_our = R.ref_simulate(fwd.encode(), m, np.asarray(ours, np.uint32).ctypes.data, k, reps, 0)
    assert abs(s_our - s_ref) / s_ref < 0.01, (s_our, s_ref)


OPIMC_EXE = os.path.join(ROOT, "oracle", "_ref", "opimc")


@pytest.mark.parametrize("eps", [0.5, 0.2])
def test_opimc_matches_reference_tool(tmp_path, eps):
    # OPIM-C (include/ripples/opimc.h:150-243) restated over the oracle
    # against the reference's own opimc tool on the 2^14-vertex IC
    # configuration: theta_0 and theta_max equal, and the spread of the two
    # seed sets, both measured by the reference's simulate, within 1%.
    R = O.reference()
    if R is None or not os.path.exists(OPIMC_EXE):
        pytest.skip("oracle/_ref not built")
    g = rb.HostGraph.rmat(14, 1 << 18, seed=0).with_weights(rb.WEIGHTS_UNIFORM, seed=1,
                                                             lo=0.0, hi=0.1)
    bwd, fwd = str(tmp_path / "g.bin"), str(tmp_path / "gf.bin")
    g.write_binary(bwd, backward=True)
    g.write_binary(fwd, backward=False)
    out = str(tmp_path / "opimc.json")
    subprocess.run([OPIMC_EXE, "-i", bwd, "--reload-binary", "-d", "IC", "-k", "20", "-e",
                    str(eps), "--delta", "0.05", "-o", out, "-p"], check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                   env=dict(os.environ, OMP_NUM_THREADS="4"), timeout=600)
    with open(out) as fh:
        rec = json.load(fh)[0]
    thr = O.pack("IC", g.index, g.weights)
    ours = O.opimc("IC", g.n, g.index, g.src, thr, 20, eps, 0.05, seed=0)
    assert ours["theta_zero"] == rec["ThetaZero"] and ours["theta_max"] == rec["ThetaMax"]
    assert len(ours["seeds"]) == len(rec["Seeds"]) == 20
    s_ref = R.ref_simulate(fwd.encode(), 0, np.asarray(rec["Seeds"], np.uint32).ctypes.data,
                           20, 3000, 0)
    s_our = R.ref_simulate(fwd.encode(), 0, np.asarray(ours["seeds"], np.uint32).ctypes.data,
                           20, 3000, 0)
    assert abs(s_our - s_ref) / s_ref < 0.01, (s_our, s_ref)


def test_opimc_oracle_arithmetic_matches_reference():
    R = O.reference()
    if R is None:
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(9)
    for _ in range(2000):
        n = int(rng.integers(100, 1 << 24))
        k = int(rng.integers(1, 200))
        eps = float(rng.choice([0.05, 0.1, 0.3]))
        d = float(rng.choice([0.05, 0.01, 0.001]))
        theta = int(rng.integers(1, 10 ** 7))
        cov = int(rng.integers(0, theta + 1))
        t0, tm, b = O.opimc_math(n, eps, k, d, cov, theta)
        assert t0 == R.ref_opimc_theta_zero(n, eps, k, d)
        assert tm == R.ref_opimc_theta_max(n, eps, k, d)
        assert np.float32(R.ref_opimc_lower_bound(cov, d, n, theta)) == b[0]
        assert np.float32(R.ref_opimc_upper_bound(cov, d, n, theta)) == b[1]
