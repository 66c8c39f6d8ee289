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
