"""Shared test setup: repository on sys.path, the `gpu` marker, golden fixtures."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on a B200 with -m gpu)")


@pytest.fixture(scope="session")
def golden_nbor():
    return np.load(os.path.join(GOLDEN, "nbor_ref.npz"))


@pytest.fixture(scope="session")
def golden_engine():
    g = np.load(os.path.join(GOLDEN, "ref_engine.npz"))
    cases = {}
    for key in g.files:
        name, field = key.split("/")
        cases.setdefault(name, {})[field] = g[key]
    return cases


def engine_case_problem(case, golden_nbor, module):
    """Problem object (oracle or product module) of one ref_engine.npz case."""
    lat = str(case["lattice"])
    ss = case["shell_size"]
    nbor = golden_nbor[lat][:, : int(ss.sum())]
    return module.Problem(nbor, ss, case["species"], case["weight"], case["target"])


def opt_call_args():
    """The positional arguments the reference driver passes to run_local_parallel_hcs_cuda
    (pyhea/model/opt.py:89-90), rebuilt with the recorded types (tests/golden/opt_call.json,
    made by tests/golden/make_golden.py opt)."""
    import json

    d = json.load(open(os.path.join(GOLDEN, "opt_call.json")))
    a = list(d["args"])
    assert d["arg_types"][5] == "list[list[ndarray(int64)]]" and d["arg_types"][8] == "ndarray(float64)"
    a[5] = [[np.asarray(shell, dtype=np.int64) for shell in site] for site in a[5]]
    a[8] = np.asarray(a[8], dtype=np.float64)
    return a
