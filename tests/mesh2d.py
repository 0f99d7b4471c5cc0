"""2D quad4 inputs of the reference's ebePCG tests (test infrastructure).

Restates, for the tests, the 2D element matrix and mesh of
tests/test-wasm-ebePCG.js:42-75 (lk2D, identical to js/optimizer-worker.js:1732-1767)
and :223-266 (setupMesh): elements numbered idx = ely + elx*nely (column-major), node
n = (nely+1)*x + y, 2 DOFs per node, the x = 0 edge fixed in both directions, and a unit
load -1 in y at the node (nelx, nely).
"""
import numpy as np


def lk2d(nu=0.3):
    k = [1 / 2 - nu / 6, 1 / 8 + nu / 8, -1 / 4 - nu / 12, -1 / 8 + 3 * nu / 8,
         -1 / 4 + nu / 12, -1 / 8 - nu / 8, nu / 6, 1 / 8 - 3 * nu / 8]
    order = [[0, 1, 2, 3, 4, 5, 6, 7], [1, 0, 7, 6, 5, 4, 3, 2], [2, 7, 0, 5, 6, 3, 4, 1],
             [3, 6, 5, 0, 7, 2, 1, 4], [4, 5, 6, 7, 0, 1, 2, 3], [5, 4, 3, 2, 1, 0, 7, 6],
             [6, 3, 4, 1, 2, 7, 0, 5], [7, 2, 1, 4, 3, 6, 5, 0]]
    scale = 1 / (1 - nu * nu)
    return np.array([[k[j] * scale for j in row] for row in order], dtype=np.float64).ravel()


def setup_mesh(nelx, nely):
    """(edofs int32[nel*8], freedofs int32, F float64[ndof]) of setupMesh."""
    nel = nelx * nely
    ndof = 2 * (nelx + 1) * (nely + 1)
    ed = np.zeros(nel * 8, np.int32)
    for ely in range(nely):
        for elx in range(nelx):
            o = (ely + elx * nely) * 8
            n1 = (nely + 1) * elx + ely
            n2 = (nely + 1) * (elx + 1) + ely
            ed[o:o + 8] = [2 * n1, 2 * n1 + 1, 2 * n2, 2 * n2 + 1, 2 * n2 + 2, 2 * n2 + 3, 2 * n1 + 2, 2 * n1 + 3]
    fixed = np.zeros(ndof, np.uint8)
    for j in range(nely + 1):
        fixed[2 * j] = fixed[2 * j + 1] = 1
    free = np.flatnonzero(fixed == 0).astype(np.int32)
    F = np.zeros(ndof)
    F[2 * ((nely + 1) * nelx + nely) + 1] = -1.0
    return ed, free, F


def scenario_densities(name, nel):
    """Density fields of the reference's 2D ebePCG tests (:286-364)."""
    if name == "solid":
        return np.ones(nel)
    if name == "graded":
        return 0.2 + 0.8 * (np.arange(nel) / nel)
    if name == "checkerboard":
        return np.where(np.arange(nel) % 2 == 0, 1.0, 0.001)
    raise ValueError(name)
