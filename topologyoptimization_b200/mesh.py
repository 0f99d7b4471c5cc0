"""Grid numbering, boundary conditions and loads of the reference's 3D worker.

Host-side input builders (index bookkeeping, no arithmetic on the solve path):
  - edofs3d            _precomputeEdofs3D       js/optimizer-worker-3d.js:1448-1494
  - fixed_dofs         getFixedDOFs/_addNodeDOFs js/optimizer-worker-3d.js:4429-4493
  - load_vector        getLoadVector            js/optimizer-worker-3d.js:4495-4547
  - constraint_elements getConstraintElements   js/optimizer-worker-3d.js:4551-4591
  - force_elements     getForceElements         js/optimizer-worker-3d.js:4596-4620
Element e = ex + ey*nelx + ez*nelx*nely; node n = x*(nely+1)*(nelz+1) + y*(nelz+1) + z.
"""
import math

import numpy as np

# local corner offsets (x, y, z) of the hex8, in the reference's order
CORNERS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                    [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.int64)


def ndof(nelx, nely, nelz):
    return 3 * (nelx + 1) * (nely + 1) * (nelz + 1)


def node_id(x, y, z, nely, nelz):
    return (np.asarray(x) * (nely + 1) + np.asarray(y)) * (nelz + 1) + np.asarray(z)


def edofs3d(nelx, nely, nelz):
    ez, ey, ex = np.meshgrid(np.arange(nelz), np.arange(nely), np.arange(nelx), indexing="ij")
    ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()  # element order: x fastest
    nodes = node_id(ex[:, None] + CORNERS[:, 0], ey[:, None] + CORNERS[:, 1], ez[:, None] + CORNERS[:, 2],
                    nely, nelz)
    ed = (3 * nodes[:, :, None] + np.arange(3)).reshape(-1, 24)
    return ed.astype(np.int32).ravel()


def _dof_mask(mode):
    if mode is None or mode == "all":
        return (True, True, True)
    return ("x" in mode, "y" in mode, "z" in mode)


def fixed_dofs(nelx, nely, nelz, position, constraint_dofs="all"):
    """List of fixed DOFs in the reference's push order."""
    mx, my, mz = _dof_mask(constraint_dofs)
    nodes = []
    if position == "left":
        nodes = [node_id(0, j, k, nely, nelz) for j in range(nely + 1) for k in range(nelz + 1)]
    elif position == "right":
        nodes = [node_id(nelx, j, k, nely, nelz) for j in range(nely + 1) for k in range(nelz + 1)]
    elif position == "bottom":
        nodes = [node_id(i, 0, k, nely, nelz) for i in range(nelx + 1) for k in range(nelz + 1)]
    elif position == "top":
        nodes = [node_id(i, nely, k, nely, nelz) for i in range(nelx + 1) for k in range(nelz + 1)]
    elif position == "bottom-corners":
        nodes = [node_id(0, 0, 0, nely, nelz), node_id(nelx, 0, 0, nely, nelz),
                 node_id(0, nely, 0, nely, nelz), node_id(nelx, nely, 0, nely, nelz)]
    out = []
    for n in nodes:
        n = int(n)
        if mx:
            out.append(3 * n)
        if my:
            out.append(3 * n + 1)
        if mz:
            out.append(3 * n + 2)
    return np.array(out, dtype=np.int64)


def fixed_mask(nelx, nely, nelz, position="left", constraint_dofs="all", fixeddofs=None):
    m = np.zeros(ndof(nelx, nely, nelz), np.uint8)
    d = fixed_dofs(nelx, nely, nelz, position, constraint_dofs) if fixeddofs is None else np.asarray(fixeddofs)
    d = d[(d >= 0) & (d < m.size)]
    m[d] = 1
    return m


def load_vector(nelx, nely, nelz, direction="down", magnitude=1.0, force_vector=None):
    """getLoadVector: a Float32Array F with one loaded node."""
    F = np.zeros(ndof(nelx, nely, nelz), np.float32)
    if force_vector is not None and len(force_vector) >= 3:
        fv = np.asarray(force_vector[:3], np.float64)
        ln = np.sqrt((fv ** 2).sum())
        if ln > 0:
            n = int(node_id(nelx, nely, nelz, nely, nelz))
            F[3 * n:3 * n + 3] = fv / ln * magnitude
        return F
    if direction in ("down", "up"):
        n = int(node_id(nelx, nely, nelz, nely, nelz))
        F[3 * n + 1] = -magnitude if direction == "down" else magnitude
    elif direction == "left":
        n = int(node_id(nelx, nely // 2, nelz // 2, nely, nelz))
        F[3 * n] = -magnitude
    elif direction == "right":
        n = int(node_id(0, nely // 2, nelz // 2, nely, nelz))
        F[3 * n] = magnitude
    elif direction == "top-center":
        n = int(node_id(nelx // 2, nely // 2, nelz, nely, nelz))
        F[3 * n + 2] = magnitude
    return F


def constraint_elements(nelx, nely, nelz, position):
    e = []
    if position == "left":
        e = [ey * nelx + ez * nelx * nely for ez in range(nelz) for ey in range(nely)]
    elif position == "right":
        e = [(nelx - 1) + ey * nelx + ez * nelx * nely for ez in range(nelz) for ey in range(nely)]
    elif position == "bottom":
        e = [ex + ez * nelx * nely for ez in range(nelz) for ex in range(nelx)]
    elif position == "top":
        e = [ex + (nely - 1) * nelx + ez * nelx * nely for ez in range(nelz) for ex in range(nelx)]
    elif position == "bottom-corners":
        e = [0, nelx - 1, (nely - 1) * nelx, (nelx - 1) + (nely - 1) * nelx]
    return np.array(e, dtype=np.int64)


def force_elements(nelx, nely, nelz, direction):
    if direction in ("down", "up"):
        return np.array([(nelx - 1) + (nely - 1) * nelx + (nelz - 1) * nelx * nely])
    if direction == "left":
        return np.array([(nelx - 1) + (nely // 2) * nelx + (nelz // 2) * nelx * nely])
    if direction == "right":
        return np.array([(nely // 2) * nelx + (nelz // 2) * nelx * nely])
    if direction == "top-center":
        return np.array([nelx // 2 + (nely // 2) * nelx + (nelz - 1) * nelx * nely])
    return np.array([], dtype=np.int64)


def structured_dims(edofs, nel, ndof_):
    """Recover (nelx, nely, nelz) when edofs is the reference's structured numbering
    (as passed by GPUFEASolver.setup, which carries no grid sizes); None otherwise."""
    ed = np.asarray(edofs).reshape(-1, 24) if len(edofs) == nel * 24 else None
    if ed is None or nel < 1 or ed[0, 0] != 0:
        return None
    nnz = int(ed[0, 9] // 3)           # node of corner (0,1,0) is nnz
    nynz = int(ed[0, 3] // 3)          # node of corner (1,0,0) is nny*nnz
    if nnz < 2 or nynz % nnz:
        return None
    nny = nynz // nnz
    if ndof_ % (3 * nynz):
        return None
    nnx = ndof_ // (3 * nynz)
    dims = (nnx - 1, nny - 1, nnz - 1)
    if dims[0] * dims[1] * dims[2] != nel or min(dims) < 1:
        return None
    if not np.array_equal(edofs3d(*dims), np.asarray(edofs, dtype=np.int32).ravel()):
        return None
    return dims


# ---- the 2D worker's mesh (js/optimizer-worker.js) ----------------------------------------
# element e = ely + elx*nely (column-major), node n = (nely+1)*x + y, DOF = 2n + {0, 1}

def ndof2d(nelx, nely):
    return 2 * (nelx + 1) * (nely + 1)


def fixed_mask2d(nelx, nely, position="left", dofs="all"):
    """getFixedDOFs (:1885-1921) as a uint8 mask."""
    m = np.zeros(ndof2d(nelx, nely), np.uint8)

    def add(n):
        if dofs == "all" or "x" in dofs:
            m[2 * n] = 1
        if dofs == "all" or "y" in dofs:
            m[2 * n + 1] = 1

    if position == "left":
        for j in range(nely + 1):
            add(j)
    elif position == "right":
        for j in range(nely + 1):
            add((nely + 1) * nelx + j)
    elif position == "bottom":
        for i in range(nelx + 1):
            add((nely + 1) * i)
    elif position == "top":
        for i in range(nelx + 1):
            add((nely + 1) * i + nely)
    return m


def load_vector2d(nelx, nely, direction="down", magnitude=1.0, force_vector=None):
    """getLoadVector (:1923-1964), float32 as the reference's Float32Array."""
    F = np.zeros(ndof2d(nelx, nely), np.float32)
    if force_vector is not None and len(force_vector) >= 2:
        ln = math.sqrt(force_vector[0] ** 2 + force_vector[1] ** 2)
        if ln > 0:
            n = (nely + 1) * nelx + nely
            F[2 * n] = force_vector[0] / ln * magnitude
            F[2 * n + 1] = force_vector[1] / ln * magnitude
        return F
    if direction == "down":
        F[2 * ((nely + 1) * nelx + nely) + 1] = -magnitude
    elif direction == "up":
        F[2 * ((nely + 1) * nelx) + 1] = magnitude
    elif direction == "left":
        F[2 * ((nely + 1) * nelx + nely // 2)] = -magnitude
    elif direction == "right":
        F[2 * (nely // 2)] = magnitude
    return F


def constraint_elements2d(nelx, nely, position):
    """getConstraintElements (:1966-1986)."""
    if position == "left":
        return list(range(nely))
    if position == "right":
        return [ey + (nelx - 1) * nely for ey in range(nely)]
    if position == "bottom":
        return [ex * nely for ex in range(nelx)]
    if position == "top":
        return [(nely - 1) + ex * nely for ex in range(nelx)]
    return []


def force_elements2d(nelx, nely, direction):
    """getForceElements (:1988-2014)."""
    if direction == "down":
        return [(nely - 1) + (nelx - 1) * nely]
    if direction == "up":
        return [(nelx - 1) * nely]
    if direction == "left":
        return [nely // 2 + (nelx - 1) * nely]
    if direction == "right":
        return [nely // 2]
    return []
