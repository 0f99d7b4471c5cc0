import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and the built libtpo.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def native():
    """libtpo on a GPU; the test fails (not skips) when the library or device is missing."""
    from topologyoptimization_b200 import _native as N
    N.lib()
    assert N.device_available(), "no sm_100 device visible to libtpo"
    return N


def rel_inf(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def cantilever_load(nelx, nely, nelz, per_node=-1.0):
    """-1 in z on every node of the line (x = nelx, y = 0..nely, z = 0)."""
    from topologyoptimization_b200 import mesh
    F = np.zeros(mesh.ndof(nelx, nely, nelz))
    for j in range(nely + 1):
        n = mesh.node_id(nelx, j, 0, nely, nelz)
        F[3 * n + 2] = per_node
    return F


def top_center_load(nelx, nely, nelz):
    """-1 in y at the top-centre node (tests/test-wasm-mgpcg.js:125-153)."""
    from topologyoptimization_b200 import mesh
    F = np.zeros(mesh.ndof(nelx, nely, nelz))
    n = mesh.node_id(nelx // 2, nely // 2, nelz, nely, nelz)
    F[3 * n + 1] = -1.0
    return F
