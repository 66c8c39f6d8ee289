import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden_selection():
    z = np.load(os.path.join(GOLDEN, "selection_cases.npz"))
    cases = []
    for i in range(int(z["num_cases"][0])):
        n, k = (int(x) for x in z[f"c{i}_meta"])
        cases.append(dict(n=n, k=k, off=z[f"c{i}_off"], vtx=z[f"c{i}_vtx"],
                          seeds=z[f"c{i}_seeds"], f=float(z[f"c{i}_f"][0])))
    return cases


@pytest.fixture(scope="session")
def golden_theta():
    with open(os.path.join(GOLDEN, "theta_values.json")) as fh:
        return json.load(fh)


@pytest.fixture(scope="session")
def golden_kat():
    with open(os.path.join(GOLDEN, "kat_counting.json")) as fh:
        return json.load(fh)


@pytest.fixture(scope="session")
def golden_wc16():
    """The reference sequential sampler's counts on R-MAT 2^16, weighted
    cascade (tests/golden/make_golden.py, WC16), with the graph rebuilt from
    its parameters by the oracle's generator."""
    from oracle import oracle as O
    z = dict(np.load(os.path.join(GOLDEN, "sampler_reference_wc16.npz")))
    scale, draws, seed = (int(x) for x in z["params"])
    n, idx, src, w = O.rmat_graph(scale, draws, seed=seed, weights="wc")
    return dict(z, n=n, index=idx, src=src, w=w, scale=scale, draws=draws, seed=seed)


def chi2_homogeneity(a, b, min_expected=20):
    """Chi-square test that two count vectors come from one distribution;
    cells with fewer than 2 * min_expected joint counts are pooled."""
    from scipy import stats
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    keep = (a + b) >= 2 * min_expected
    table = np.vstack([np.append(a[keep], a[~keep].sum()), np.append(b[keep], b[~keep].sum())])
    table = table[:, table.sum(axis=0) > 0]
    chi2, p, dof, _ = stats.chi2_contingency(table)
    return chi2, p, dof


def assert_same_distribution(freq, sizes, ref_freq, ref_size_hist):
    """North-star check 3: per-vertex occurrence frequencies within a
    chi-square bound (p > 1e-4) and mean RRR size within 1% of the reference
    sampler's."""
    chi2, p, dof = chi2_homogeneity(freq, ref_freq)
    assert p > 1e-4, (chi2, dof, p)
    hist = np.asarray(ref_size_hist, np.float64)
    ref_mean = (hist * np.arange(len(hist))).sum() / hist.sum()
    mean = float(np.mean(sizes))
    assert abs(mean - ref_mean) / ref_mean < 0.01, (mean, ref_mean)


@pytest.fixture(scope="session")
def golden_sampler():
    return dict(np.load(os.path.join(GOLDEN, "sampler_reference.npz")))


def karate(weight=None):
    import ripples_b200 as rb
    e = np.loadtxt(os.path.join(GOLDEN, "karate.tsv"), dtype=np.float64)
    w = e[:, 2].astype(np.float32) if weight is None else np.full(len(e), weight, np.float32)
    return rb.HostGraph.from_edges(34, e[:, 0].astype(np.int64) - 1,
                                   e[:, 1].astype(np.int64) - 1, w)


def csr_of(sets):
    off = np.zeros(len(sets) + 1, np.uint64)
    off[1:] = np.cumsum([len(s) for s in sets])
    vtx = np.concatenate([np.asarray(s, np.uint32) for s in sets]) if sets else np.zeros(0, np.uint32)
    return off, vtx


@pytest.fixture(scope="session")
def ctx():
    import ripples_b200 as rb
    c = rb.Context(0)
    yield c
    c.close()
