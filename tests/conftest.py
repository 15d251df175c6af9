import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


@pytest.fixture(scope="session")
def small_workload():
    """config0 set-up with 2,000 particles (mesh and fields at full size)."""
    from pyrticle_b200 import problems
    return problems.make("config0", scale=0.2)


@pytest.fixture(scope="session")
def oracle_mesh(small_workload):
    from oracle import pyoracle
    from pyrticle_b200 import meshgen
    w = small_workload
    return pyoracle.OracleMesh(w.mesh, w.nodes, meshgen.element_bins(w.mesh))
