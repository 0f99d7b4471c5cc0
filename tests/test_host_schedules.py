"""Host-side loop control of TopologyOptimizerWorker3D (no device): the CG tolerance
schedule of FE (js/optimizer-worker-3d.js:4189-4193) and the load cases of getLoadVector
(:4495-4547)."""
import math

import numpy as np

from topologyoptimization_b200 import mesh
from topologyoptimization_b200.worker3d import cg_tolerance


def test_cg_tolerance_schedule():
    # exp(log 1e-3 + progress (log 1e-8 - log 1e-3)), progress = (iter - 1) / (maxIter - 1)
    for n in (2, 5, 51, 300):
        assert math.isclose(cg_tolerance(1, n), 1e-3, rel_tol=1e-14)
        assert math.isclose(cg_tolerance(n, n), 1e-8, rel_tol=1e-14)
        tols = [cg_tolerance(i, n) for i in range(1, n + 1)]
        assert all(a > b for a, b in zip(tols, tols[1:]))  # strictly decreasing
        ratios = [b / a for a, b in zip(tols, tols[1:])]
        assert max(ratios) - min(ratios) < 1e-12  # geometric
    assert math.isclose(cg_tolerance(26, 51), math.sqrt(1e-3 * 1e-8), rel_tol=1e-14)
    assert math.isclose(cg_tolerance(1, 1), 1e-8, rel_tol=1e-14)  # one iteration: the final tolerance


def test_load_vector_cases():
    nelx, nely, nelz = 6, 4, 2
    nd = mesh.ndof(nelx, nely, nelz)
    cases = {
        "down": (mesh.node_id(nelx, nely, nelz, nely, nelz), 1, -1.0),
        "up": (mesh.node_id(nelx, nely, nelz, nely, nelz), 1, 1.0),
        "left": (mesh.node_id(nelx, nely // 2, nelz // 2, nely, nelz), 0, -1.0),
        "right": (mesh.node_id(0, nely // 2, nelz // 2, nely, nelz), 0, 1.0),
        "top-center": (mesh.node_id(nelx // 2, nely // 2, nelz, nely, nelz), 2, 1.0),
    }
    for direction, (node, comp, sign) in cases.items():
        F = mesh.load_vector(nelx, nely, nelz, direction, magnitude=2.5)
        assert F.dtype == np.float32 and F.size == nd
        assert np.count_nonzero(F) == 1
        assert F[3 * int(node) + comp] == np.float32(2.5 * sign)
    # an explicit force vector is normalised and applied at the far corner node
    F = mesh.load_vector(nelx, nely, nelz, force_vector=[3.0, 0.0, 4.0], magnitude=10.0)
    n = int(mesh.node_id(nelx, nely, nelz, nely, nelz))
    assert np.array_equal(F[3 * n:3 * n + 3], np.array([6.0, 0.0, 8.0], np.float32))
    assert np.count_nonzero(F) == 2
