import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA library")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    """Builds the CPU oracle (and the reference's CPU code when its sources are present)."""
    import oracle

    if not os.path.exists(oracle.ORACLE_SO) or (os.path.isdir(os.path.join(oracle.REF_SRC, "serial"))
                                                and not oracle.ref_available()):
        oracle.build()
    yield


def load_golden_json():
    import json

    with open(os.path.join(GOLDEN, "reference_tests.json")) as f:
        return json.load(f)


def golden_mesh(g, dtype=np.float64):
    from ssdf_b200.workloads import Mesh

    v = np.stack([np.asarray(g["sx"]), np.asarray(g["sy"]), np.asarray(g["sz"])], 1).astype(dtype)
    t = np.stack([g["s0"], g["s1"], g["s2"]], 1).astype(np.int32)
    return Mesh(v.astype(np.float64), t)
