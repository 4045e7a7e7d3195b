import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle.reference_dir import REFERENCE_DIR, reference_dir  # noqa: E402

REFERENCE = REFERENCE_DIR
WIKI = os.path.join(REFERENCE, "examples", "Sample-Graph-Wiki-Vote.txt")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (run with -m gpu)")
    config.addinivalue_line("markers", "slow: larger CPU cases")


@pytest.fixture(scope="session")
def golden():
    z = np.load(os.path.join(ROOT, "tests", "golden", "golden.npz"))
    g = {k: z[k] for k in z.files}
    g["meta"] = json.loads(bytes(g["meta"]).decode())
    return g


@pytest.fixture(scope="session")
def has_reference():
    return reference_dir() is not None


@pytest.fixture(scope="session")
def engine():
    from kites_b200 import capi

    eng = capi.Engine(0)
    yield eng
    eng.close()


@pytest.fixture(scope="session")
def cfg1_edges(golden):
    from kites_b200 import capi

    c = golden["meta"]["cfg1"]
    return capi.gen_rmat(c["scale"], c["n_edges"], c["a"], c["b"], c["c"], c["seed"],
                         c["w_lo"], c["w_hi"], n_vertices=c["n_vertices"])
