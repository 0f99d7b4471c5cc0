"""Pins of the CPU oracle against the reference's own known-answer tests and against an
independent scipy assembly.  The reference (JavaScript/WebAssembly) cannot run in
this environment, so these are the anchors of every parity claim:

  - tests/test-fea-benchmarks.js:295-357   Ke symmetry and rigid-body null space (2D
                                           there; the 3D equivalents here)
  - tests/test-fea-benchmarks.js:410-426,
    :590, :753                             patch test, energy balance, Poisson ratio
  - tests/test-wasm-applyA.js:176-341      applyA scenarios (synthetic Ke, 1^3..6^3,
                                           partial activity, zero input, no actives)
  - tests/test-wasm-mgpcg.js:607-695       MGPCG 4^3 / 6^3 / graded, zero force
  - tests/golden/*.npz                     fixtures written by tests/golden/make_golden.py
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from conftest import rel_inf, top_center_load

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def independent_ke(nu):
    """Hex8 Ke from the textbook B^T C B Gauss sum, written independently in numpy."""
    f = 1.0 / ((1 + nu) * (1 - 2 * nu))
    C = np.zeros((6, 6))
    C[:3, :3] = f * nu
    np.fill_diagonal(C[:3, :3], f * (1 - nu))
    C[3:, 3:] = np.eye(3) * f * (1 - 2 * nu) / 2
    corners = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                        [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)
    K = np.zeros((24, 24))
    g = 1 / np.sqrt(3)
    for xi in (-g, g):
        for eta in (-g, g):
            for zeta in (-g, g):
                q = np.array([xi, eta, zeta])
                # dN/dxi for N = prod(1 + c_k q_k)/8, times the Jacobian 1/0.5 ... the
                # reference uses dN*0.125 with J = I; keep its convention
                dN = np.zeros((8, 3))
                for a, c in enumerate(corners):
                    for k in range(3):
                        t = c[k]
                        for m in range(3):
                            if m != k:
                                t *= 1 + c[m] * q[m]
                        dN[a, k] = t * 0.125
                B = np.zeros((6, 24))
                B[0, 0::3] = dN[:, 0]
                B[1, 1::3] = dN[:, 1]
                B[2, 2::3] = dN[:, 2]
                B[3, 0::3] = dN[:, 1]
                B[3, 1::3] = dN[:, 0]
                B[4, 1::3] = dN[:, 2]
                B[4, 2::3] = dN[:, 1]
                B[5, 0::3] = dN[:, 2]
                B[5, 2::3] = dN[:, 0]
                K += B.T @ C @ B
    return K


def assemble(O, nelx, nely, nelz, E, Ke):
    ed = O.edofs3d(nelx, nely, nelz).reshape(-1, 24)
    nd = O.ndof_of(nelx, nely, nelz)
    rows = np.repeat(ed, 24, axis=1).ravel()
    cols = np.tile(ed, (1, 24)).ravel()
    vals = (E[:, None, None] * Ke.reshape(24, 24)[None]).ravel()
    return sp.csr_matrix((vals, (rows, cols)), shape=(nd, nd))


def rigid_modes():
    X = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    R = []
    for d in range(3):
        v = np.zeros(24)
        v[d::3] = 1
        R.append(v)
    for a, b in ((0, 1), (1, 2), (0, 2)):
        v = np.zeros(24)
        v[a::3] = -X[:, b]
        v[b::3] = X[:, a]
        R.append(v)
    return R


@pytest.mark.parametrize("nu", [0.3, 0.25, 0.45])
def test_ke_properties(oracle, nu):
    Ke = oracle.lk(nu).reshape(24, 24)
    assert np.abs(Ke - Ke.T).max() < 1e-15
    for r in rigid_modes():
        assert np.abs(Ke @ r).max() < 1e-12
    ev = np.linalg.eigvalsh((Ke + Ke.T) / 2)
    assert ev.min() > -1e-12
    assert np.linalg.matrix_rank(Ke, 1e-10) == 18
    assert np.abs(Ke - independent_ke(nu)).max() < 1e-14


def test_ke_golden(oracle):
    g = np.load(os.path.join(GOLDEN, "ke_nu0.3.npz"))
    assert np.array_equal(oracle.lk(0.3), g["Ke"])


def test_mesh_builders_match(oracle):
    from topologyoptimization_b200 import mesh
    for dims in [(1, 1, 1), (3, 2, 4), (5, 3, 2)]:
        assert np.array_equal(oracle.edofs3d(*dims), mesh.edofs3d(*dims))
        for pos in ["left", "right", "bottom", "top", "bottom-corners"]:
            assert np.array_equal(oracle.fixed_mask(*dims, pos), mesh.fixed_mask(*dims, pos))
            m = np.zeros(np.prod(dims), np.uint8)
            m[mesh.constraint_elements(*dims, pos)] = 1
            assert np.array_equal(oracle.constraint_elements(*dims, pos), m)
        nd = mesh.ndof(*dims)
        assert mesh.structured_dims(mesh.edofs3d(*dims), int(np.prod(dims)), nd) == dims
    scrambled = mesh.edofs3d(3, 2, 2).copy()
    scrambled[[0, 1]] = scrambled[[1, 0]]
    assert mesh.structured_dims(scrambled, 12, mesh.ndof(3, 2, 2)) is None


def test_apply_matches_assembly(oracle):
    rng = np.random.default_rng(7)
    nelx, nely, nelz = 5, 3, 4
    Ke = oracle.lk(0.3)
    x = rng.uniform(1e-3, 1, nelx * nely * nelz)
    E = 1e-9 + x ** 3 * (1 - 1e-9)
    active = np.flatnonzero(E > 1e-6).astype(np.int32)
    Eact = np.where(E > 1e-6, E, 0.0)
    p = rng.standard_normal(oracle.ndof_of(nelx, nely, nelz))
    Ap = oracle.apply_a(Ke, oracle.edofs3d(nelx, nely, nelz), E, active, p)
    K = assemble(oracle, nelx, nely, nelz, Eact, Ke)
    assert rel_inf(Ap, K @ p) < 1e-13


def synthetic_ke():
    """makeSimpleKE, tests/test-wasm-applyA.js:77-88."""
    K = np.zeros((24, 24))
    for i in range(24):
        K[i, i] = 10.0 + i
        if i + 1 < 24:
            K[i, i + 1] = -1.0
            K[i + 1, i] = -1.0
    return K.ravel()


@pytest.mark.parametrize("dims,frac", [((1, 1, 1), 1.0), ((3, 3, 3), 1.0), ((4, 4, 4), 0.5), ((2, 2, 2), 1.0),
                                       ((6, 6, 6), 1.0)])
def test_apply_reference_scenarios(oracle, dims, frac):
    rng = np.random.default_rng(11)
    nel = int(np.prod(dims))
    nd = oracle.ndof_of(*dims)
    Ke = synthetic_ke()
    ed = oracle.edofs3d(*dims)
    E = rng.uniform(0.1, 1.0, nel)
    active = np.arange(nel, dtype=np.int32)[: max(1, int(nel * frac))]
    p = rng.standard_normal(nd)
    Ap = oracle.apply_a(Ke, ed, E, active, p)
    Eact = np.zeros(nel)
    Eact[active] = E[active]
    assert rel_inf(Ap, assemble(oracle, *dims, Eact, Ke) @ p) < 1e-13
    assert not np.any(oracle.apply_a(Ke, ed, E, active, np.zeros(nd)))
    assert not np.any(oracle.apply_a(Ke, ed, E, np.zeros(0, np.int32), p))


def test_dense_matvec(oracle):
    rng = np.random.default_rng(3)
    K = rng.standard_normal((50, 50))
    p = rng.standard_normal(50)
    assert rel_inf(oracle.dense_matvec(K, p), K @ p) < 1e-14


def direct(oracle, dims, x, F, fixed, penal=3.0):
    Ke = oracle.lk(0.3)
    E = 1e-9 + x.astype(np.float64) ** penal * (1 - 1e-9)
    E = np.where(E > 1e-6, E, 0.0)
    K = assemble(oracle, *dims, E, Ke)
    free = np.flatnonzero(fixed == 0)
    u = np.zeros(len(F))
    u[free] = spl.spsolve(K[free][:, free].tocsc(), F[free])
    return u, K


@pytest.mark.parametrize("dims,graded", [((4, 4, 4), False), ((6, 6, 6), False), ((4, 4, 4), True)])
def test_mgpcg_reference_scenarios(oracle, dims, graded):
    nel = int(np.prod(dims))
    fixed = oracle.fixed_mask(*dims, "bottom-corners")
    F = top_center_load(*dims)
    x = (0.3 + 0.7 * np.arange(nel) / nel) if graded else np.ones(nel)
    x = x.astype(np.float32)
    u, K = direct(oracle, dims, x, F, fixed)
    mg = oracle.MG(*dims, oracle.lk(0.3), fixed)
    mg.update(x, 3.0)
    U, it = mg.mgpcg(F, 500, 1e-6)
    assert 0 < it < 500
    assert rel_inf(U, u) < 1e-4
    assert abs(F @ U - F @ u) / abs(F @ u) < 1e-3
    U0, it0 = mg.mgpcg(np.zeros_like(F), 500, 1e-6)
    assert it0 == 0 and not np.any(U0)


def test_ebe_pcg_and_energy_balance(oracle):
    dims = (8, 4, 4)
    rng = np.random.default_rng(5)
    nel = int(np.prod(dims))
    x = rng.uniform(0.2, 1.0, nel).astype(np.float32)
    fixed = oracle.fixed_mask(*dims, "left")
    F = top_center_load(*dims) * 1e3
    u, K = direct(oracle, dims, x, F, fixed)
    free = np.flatnonzero(fixed == 0).astype(np.int32)
    U, it = oracle.ebe_pcg(x.astype(np.float64), oracle.lk(0.3), oracle.edofs3d(*dims), F, np.zeros(len(F)), free,
                           len(F), 1e-9, 1.0, 3.0, 5000, 1e-10)
    assert it < 5000
    assert rel_inf(U, u) < 1e-7
    assert abs(U @ (K @ U) - F @ U) / abs(F @ U) < 1e-8


def test_patch_and_poisson(oracle):
    """Uniform traction on a roller-supported block: exact uniform strain (patch test,
    tests/test-fea-benchmarks.js:410-426) and the Poisson ratio -eps_y/eps_x = nu (:753)."""
    nelx, nely, nelz = 6, 3, 3
    nu = 0.3
    from topologyoptimization_b200 import mesh
    nd = mesh.ndof(nelx, nely, nelz)
    fixed = np.zeros(nd, np.uint8)
    F = np.zeros(nd)
    for i in range(nelx + 1):
        for j in range(nely + 1):
            for k in range(nelz + 1):
                n = mesh.node_id(i, j, k, nely, nelz)
                if i == 0:
                    fixed[3 * n] = 1
                if j == 0:
                    fixed[3 * n + 1] = 1
                if k == 0:
                    fixed[3 * n + 2] = 1
                if i == nelx:  # consistent nodal forces of a unit traction
                    wy = 0.5 if j in (0, nely) else 1.0
                    wz = 0.5 if k in (0, nelz) else 1.0
                    F[3 * n] = wy * wz
    x = np.ones(nelx * nely * nelz, np.float32)
    u, _ = direct(oracle, (nelx, nely, nelz), x, F, fixed)
    mg = oracle.MG(nelx, nely, nelz, oracle.lk(nu), fixed)
    mg.update(x, 3.0)
    U, it = mg.fe_pcg(F, np.zeros(nd), 2000, 1e-10, precond="jacobi")
    # lk() integrates in natural coordinates with J = I, so its Ke is twice the
    # stiffness of a unit cube: the block responds with an effective modulus of 2.
    E = 2.0
    for i in range(nelx + 1):
        for j in range(nely + 1):
            for k in range(nelz + 1):
                n = mesh.node_id(i, j, k, nely, nelz)
                assert abs(U[3 * n] - i / E) < 1e-6
                assert abs(U[3 * n + 1] + nu * j / E) < 1e-6
                assert abs(U[3 * n + 2] + nu * k / E) < 1e-6
    # the reference's absolute 1e-12 shift in alpha/beta stalls CG near 1e-8 here
    assert rel_inf(U, u) < 1e-7


def test_vcycle_is_symmetric(oracle):
    dims = (8, 4, 4)
    rng = np.random.default_rng(2)
    nel = int(np.prod(dims))
    fixed = oracle.fixed_mask(*dims, "left")
    mg = oracle.MG(*dims, oracle.lk(0.3), fixed)
    mg.update(rng.uniform(0.2, 1, nel).astype(np.float32), 3.0)
    a = rng.standard_normal(len(fixed)) * (fixed == 0)
    b = rng.standard_normal(len(fixed)) * (fixed == 0)
    assert abs(a @ mg.vcycle(b) - b @ mg.vcycle(a)) < 1e-10 * abs(a @ mg.vcycle(a))


def _void_design(dims, seed=0):
    """Densities with half the elements void (1e-3, below the 1000 Emin activity threshold)
    and a solid x = 0 layer: nodes held by a single active element appear."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    x = rng.uniform(0.2, 1.0, nx * ny * nz).astype(np.float32)
    x[rng.random(x.size) < 0.5] = 1e-3
    x.reshape(nz, ny, nx)[:, :, 0] = 1.0
    x.reshape(nz, ny, nx)[0, :, nx - 1] = 1.0  # the elements under the loaded line stay solid
    return x


def _vcycle_matrix(oracle, dims, x, **opts):
    fixed = oracle.fixed_mask(*dims, "left")
    free = np.flatnonzero(fixed == 0)
    mg = oracle.MG(*dims, oracle.lk(0.3), fixed, max_levels=3, **opts)
    mg.update(x, 3.0)
    B = np.zeros((len(free), len(free)))
    e = np.zeros(len(fixed))
    for k, i in enumerate(free):
        e[:] = 0.0
        e[i] = 1.0
        B[:, k] = mg.vcycle(e)[free]
    return B


@pytest.mark.parametrize("coarse_direct", [0, 1])
def test_safe_omega_keeps_vcycle_positive(oracle, coarse_direct):
    """Damped Jacobi with omega = 0.5 diverges where lambda_max(D^-1 A) > 4, which happens
    once a node is held by a single active element (lambda_max(diag(Ke)^-1 Ke) = 5.318 for
    nu = 0.3): the reference V-cycle is then indefinite and PCG can stall.  The per-level
    damping min(omega, 1.9 / bound) keeps it positive semidefinite (zero only on DOFs
    without stiffness)."""
    dims = (8, 4, 4)
    x = _void_design(dims)
    B = _vcycle_matrix(oracle, dims, x, coarse_direct=coarse_direct)
    Bs = _vcycle_matrix(oracle, dims, x, coarse_direct=coarse_direct, safe_omega=1)
    assert np.abs(Bs - Bs.T).max() < 1e-12 * np.abs(Bs).max()
    ev = np.linalg.eigvalsh(B)
    evs = np.linalg.eigvalsh(Bs)
    if coarse_direct == 0:
        assert ev.min() < -1e-6 * ev.max()  # the reference damping: indefinite on this design
    assert evs.min() > -1e-10 * evs.max()


def test_filter_weights(oracle):
    n = 5
    hs = oracle.filter_hs(n, n, n, 1.5)
    centre = 2 + 2 * n + 2 * n * n
    assert abs(hs[centre] - (1.5 + 6 * 0.5 + 12 * (1.5 - np.sqrt(2)))) < 1e-6
    hs2 = oracle.filter_hs(n, n, n, 2.0)
    expect = 2.0 + 6 * 1.0 + 12 * (2 - np.sqrt(2)) + 8 * (2 - np.sqrt(3))
    assert abs(hs2[centre] - expect) < 1e-5
    x = np.full(n ** 3, 0.5, np.float32)
    dc = np.full(n ** 3, -2.0, np.float32)
    dcn = oracle.filter_sens(n, n, n, 1.5, hs, x, dc)
    assert np.allclose(dcn, -2.0, rtol=1e-6)


def test_density_filter_constant(oracle):
    d = np.full(4 * 3 * 5, 0.7)
    assert np.allclose(oracle.density_filter(d, 4, 3, 5, 1.5), 0.7, rtol=1e-15)


def test_oc_volume_and_moves(oracle):
    rng = np.random.default_rng(4)
    n = 1000
    x = rng.uniform(0.1, 0.9, n).astype(np.float32)
    dc = -rng.uniform(0.01, 5.0, n).astype(np.float32)
    xnew, lmid, nb = oracle.oc(x, 0.4, dc)
    assert 20 < nb < 80
    assert abs(xnew.astype(np.float64).sum() - 0.4 * n) / n < 2e-3
    assert np.all(xnew >= np.maximum(0, x - 0.2) - 1e-7)
    assert np.all(xnew <= np.minimum(1, x + 0.2) + 1e-7)


def test_simp_small_run(oracle):
    dims = (12, 4, 4)
    fixed = oracle.fixed_mask(*dims, "left")
    from conftest import cantilever_load
    F = cantilever_load(*dims).astype(np.float32)
    pres = oracle.constraint_elements(*dims, "left")
    r = oracle.simp(*dims, F, fixed, preserved=pres, max_iter=12, solver=1, penal_start=3.0, use_projection=0,
                    cg_tol=1e-8, cg_max_iter=400, stop_on_change=1)
    c = r["compliance"]
    assert r["iterations"] == 12
    assert c[-1] < c[0]
    assert abs(r["x"].astype(np.float64).mean() - 0.3) < 0.01 + pres.mean()
