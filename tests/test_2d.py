"""The 2D worker's hot path (js/optimizer-worker.js, TopologyOptimizerWorker): its quad
element matrix, numbering, Jacobi-PCG with the absolute stopping test, energies,
sensitivities, 2D sensitivity filter, OC and change, as one device-resident SIMP step per
iteration, against the oracle's restatement of the 2D loop."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_lk2d_properties(oracle):
    """tests/test-fea-benchmarks.js:280-357 (2D): KE symmetric (< 1e-15), positive diagonal,
    translations and the rigid rotation in its null space (< 1e-12); the same matrix as the
    reference test's lk2D (tests/test-wasm-ebePCG.js:42-70)."""
    from mesh2d import lk2d
    Ke = oracle.lk2d(0.3).reshape(8, 8)
    assert np.array_equal(Ke.ravel(), lk2d(0.3))
    assert np.abs(Ke - Ke.T).max() < 1e-15
    assert (np.diag(Ke) > 0).all()
    ux = np.array([1, 0, 1, 0, 1, 0, 1, 0.0])
    uy = np.array([0, 1, 0, 1, 0, 1, 0, 1.0])
    nodes = [(0, 0), (1, 0), (1, 1), (0, 1)]
    urot = np.array([v for (nx, ny) in nodes for v in (-(ny - 0.5), nx - 0.5)])
    for u in (ux, uy, urot):
        assert np.abs(Ke @ u).sum() < 1e-12


def test_mesh2d_builders(oracle):
    """The 2D numbering of _precomputeEdofs2D (:247-268) and the reference test's setupMesh
    agree; getFixedDOFs 'left' fixes both DOFs of the x = 0 edge."""
    from mesh2d import setup_mesh
    from topologyoptimization_b200 import mesh
    import ctypes as C
    for nx, ny in ((5, 5), (20, 10), (7, 3)):
        ed_ref, free, F = setup_mesh(nx, ny)
        ed = np.zeros(nx * ny * 8, np.int32)
        oracle.lib().orc_edofs2d(nx, ny, ed.ctypes.data_as(C.c_void_p))
        assert np.array_equal(ed, ed_ref)
        fixed = mesh.fixed_mask2d(nx, ny, "left")
        assert np.array_equal(np.flatnonzero(fixed == 0), free)
        assert np.array_equal(mesh.load_vector2d(nx, ny, "down"), F.astype(np.float32))


@pytest.mark.gpu
def test_lk2d_device(native, oracle):
    from topologyoptimization_b200.worker2d import lk2d
    assert np.array_equal(lk2d(0.3), oracle.lk2d(0.3))


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(40, 40), (60, 20)])
def test_2d_simp_run(native, dims):
    """The 2D worker's loop on the device against the oracle's run (fixtures from
    tests/golden/make_golden.py): a cantilever with the x = 0 edge fixed and a unit
    downward load at the bottom-right node, penal 3, no projection, 40 iterations or the
    change stop, the worker's CG tolerance max(1e-8, change * 1e-2) with the absolute test.

    40x40 converges (change <= 0.01 at iteration 34): the same CG iteration counts
    throughout, compliance history within 1e-7 relative, final densities within 1e-5.
    60x20 does not converge in 40 iterations, and its loose absolute CG tolerance
    (about 1e-3 in ||r||) stops every solve far from convergence: the compliance of an
    unconverged CG iterate carries the rounding of the dot products (a fixed tree on the
    device, sequential in the oracle) amplified by CG's loss of orthogonality, 1.5e-6
    after 27 iterations, and it leaves the stopping iteration of a solve one rounding
    away from flipping: once a CG count differs by one the designs separate.  There the
    histories must agree within 1e-5 up to the first differing CG count (at iteration 10
    or later), and the final compliance within 1e-2."""
    from topologyoptimization_b200.worker2d import TopologyOptimizerWorker
    nx, ny = dims
    g = np.load(os.path.join(GOLDEN, f"simp2d_{nx}x{ny}.npz"))
    w = TopologyOptimizerWorker()
    r = w.optimize({"nx": nx, "ny": ny}, dict(volumeFraction=0.3, maxIterations=40, penaltyFactor=3.0, filterRadius=1.5,
                                              penalStart=3.0, useProjection=False, constraintPosition="left",
                                              forceDirection="down", preservedElements=g["preserved"].astype(bool)))
    assert r["iterations"] == len(g["compliance"])
    dc = np.abs(r["complianceHistory"] / g["compliance"] - 1)
    dx = np.abs(r["densities2D"] - g["x"]).max()
    diff = np.flatnonzero(r["cgIterations"] != g["cg"])
    first = int(diff[0]) if diff.size else len(dc)
    print(f"2D {nx}x{ny}: compliance rel max {dc.max():.3e} (first {first} iterations {dc[:first].max():.3e}), "
          f"x max abs {dx:.3e}, first differing CG count at {first}")
    assert np.array_equal(r["densities"].reshape(ny, nx), r["densities2D"].reshape(nx, ny).T)
    if dims == (40, 40):
        assert first == len(dc)
        assert dc.max() < 1e-7
        assert dx < 1e-5
    else:
        assert first >= 10
        assert dc[:first].max() < 1e-5
        assert dc[-1] < 1e-2


@pytest.mark.gpu
def test_2d_bottom_support_side_load(native, oracle):
    """Another support and load of the 2D worker: the y = 0 edge fixed ('bottom',
    getFixedDOFs :1885-1921) and the 'right' load (getLoadVector :1923-1964), their
    elements preserved, penal 3, no projection, 30 iterations or the change stop, against
    the oracle's 2D loop run here.  The run converges (change <= 0.01) in 13 iterations
    with the oracle's CG counts throughout; compliance history within 1e-9 relative
    (measured on a B200: 3.5e-11)."""
    from topologyoptimization_b200 import mesh
    from topologyoptimization_b200.worker2d import TopologyOptimizerWorker
    nx, ny = 40, 20
    fixed = mesh.fixed_mask2d(nx, ny, "bottom")
    F = mesh.load_vector2d(nx, ny, "right")
    pres = np.zeros(nx * ny, np.uint8)
    pres[mesh.constraint_elements2d(nx, ny, "bottom")] = 1
    pres[mesh.force_elements2d(nx, ny, "right")] = 1
    ro = oracle.simp2d(nx, ny, F, fixed, pres, None, max_iter=30, use_projection=0, penal_start=3.0)
    w = TopologyOptimizerWorker()
    r = w.optimize({"nx": nx, "ny": ny}, dict(volumeFraction=0.3, maxIterations=30, penaltyFactor=3.0, filterRadius=1.5,
                                              penalStart=3.0, useProjection=False, constraintPosition="bottom",
                                              forceDirection="right"))
    n = min(len(ro["compliance"]), int(r["iterations"]))
    dc = np.abs(r["complianceHistory"][:n] / ro["compliance"][:n] - 1)
    diff = np.flatnonzero(np.asarray(r["cgIterations"][:n]) != ro["cg"][:n])
    first = int(diff[0]) if diff.size else n
    print(f"2D bottom/right: iterations {r['iterations']} vs {ro['iterations']}, compliance rel max {dc.max():.3e} "
          f"(first {first}: {dc[:first].max():.3e}), first differing CG count at {first}")
    assert r["iterations"] == ro["iterations"]
    assert first == n
    assert dc.max() < 1e-9
