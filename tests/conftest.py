import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden_manifest():
    import json
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def load_case(name):
    """Inputs of a golden case: base, queries, NSGGraph, true-NN ids."""
    from parallel_anns_b200 import formats as fm
    d = os.path.join(GOLDEN, name)
    base = fm.read_fvecs(os.path.join(d, "base.fvecs"))
    q = fm.read_fvecs(os.path.join(d, "query.fvecs"))
    g = fm.read_nsg(os.path.join(d, "graph.nsg"))
    tid, _ = fm.read_true_nn(os.path.join(d, "truenn.bin"))
    return base, q, g, tid


def golden_ids(name, form, K):
    import numpy as np
    return np.fromfile(os.path.join(GOLDEN, name, form + ".ids"), dtype=np.uint32).reshape(-1, K)
