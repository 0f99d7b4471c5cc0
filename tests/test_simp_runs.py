"""Whole SIMP runs of the worker (TopologyOptimizerWorker3D.optimize,
js/optimizer-worker-3d.js:1605-2352) on the device against the oracle's runs of the
same loop (tests/golden/make_golden.py).

Every step of the device loop is checked piecewise elsewhere (bit-exact filter and OC,
float-rounding-class energy and sensitivity, converged solves at 1e-10).  Over a whole
run the solver's stopping point feeds back into the design, so the tolerances below
are those a run reaches, stated per test."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _run(nx, ny, nz, g, **cfg):
    from topologyoptimization_b200 import TopologyOptimizerWorker3D
    w = TopologyOptimizerWorker3D()
    base = dict(volumeFraction=0.3, penaltyFactor=3.0, filterRadius=1.5, constraintPosition="left", F=g["F"],
                preservedElements=g["preserved"].astype(bool))
    base.update(cfg)
    try:
        return w.optimize({"nx": nx, "ny": ny, "nz": nz}, base)
    finally:
        w.close()


def test_plain_cantilever_30x10x10_jacobi(native):
    """The plain SIMP cantilever: 30x10x10, penal 3, no projection, volfrac 0.3, rmin
    1.5, x0 = 0.3, 50 OC iterations, Jacobi-PCG at the fixed tolerance 1e-8 with a
    2000-iteration cap (the reference's ebePCG semantics, warm start).  From the fifth
    iteration on the reference's shifted recurrence stops at the cap (its 1e-12 shift
    dominates once rz < 1e-12), in the oracle and here alike, with the same iteration
    counts throughout.  Stated agreement over the 50 iterations (measured on a B200:
    4.1e-9 and 2.4e-7): compliance history within 1e-8 relative (the first iteration
    within 1e-10), final densities within 1e-6."""
    g = np.load(os.path.join(GOLDEN, "simp_30x10x10_jacobi.npz"))
    r = _run(30, 10, 10, g, maxIterations=50, penalStart=3.0, useProjection=False, linearSolver="cg",
             cgTolerance=1e-8, cgMaxIterations=2000)
    assert r["iterations"] == len(g["compliance"]) == 50
    dc = np.abs(r["complianceHistory"] / g["compliance"] - 1)
    dx = np.abs(r["densities"] - g["x"]).max()
    print(f"config0: compliance rel max {dc.max():.3e} (first {dc[0]:.3e}), x max abs {dx:.3e}, "
          f"cg {list(r['cgIterations'][:6])} vs {list(g['cg'][:6])}")
    assert np.array_equal(r["cgIterations"], g["cg"])
    assert dc[0] < 1e-10
    assert dc.max() < 1e-8
    assert dx < 1e-6


def test_worker_defaults_16x8x8(native):
    """The worker's defaults (tolerance schedule 1e-3 -> 1e-8, Heaviside projection with
    beta doubling every 5 iterations, penal continuation 1.5 -> 3, ebeMGPCG with the
    reference hierarchy capped at 400 iterations) for 20 iterations on 16x8x8, with the same
    iteration counts.  Stated agreement (measured on a B200: 2.0e-8 and 4.2e-7):
    compliance history within 1e-7 relative, final densities within 1e-5."""
    g = np.load(os.path.join(GOLDEN, "simp_16x8x8_defaults.npz"))
    r = _run(16, 8, 8, g, maxIterations=20, linearSolver="mgpcg")
    assert r["iterations"] == len(g["compliance"])
    dc = np.abs(r["complianceHistory"] / g["compliance"] - 1)
    dx = np.abs(r["densities"] - g["x"]).max()
    print(f"defaults: compliance rel max {dc.max():.3e}, x max abs {dx:.3e}, cg {list(r['cgIterations'])} vs "
          f"{list(g['cg'])}")
    assert np.array_equal(r["cgIterations"], g["cg"])
    assert dc.max() < 1e-7
    assert dx < 1e-5


def test_worker_defaults_corner_supports_12x12x6(native, oracle):
    """The worker's defaults with the other built-in supports and load: the four bottom
    corners fixed ('bottom-corners', getFixedDOFs :4478-4489) and the 'top-center' load
    (getLoadVector :4536-4540), their elements preserved, ebeMGPCG with the reference
    hierarchy, 12 iterations, against the oracle's loop run here.  Same CG counts,
    compliance history within 1e-10 relative, final densities within 1e-6 (measured on a
    B200: 1.8e-13 and bit-identical densities)."""
    from topologyoptimization_b200 import mesh
    dims = (12, 12, 6)
    fixed = mesh.fixed_mask(*dims, "bottom-corners")
    F = mesh.load_vector(*dims, "top-center")
    pres = np.zeros(int(np.prod(dims)), np.uint8)
    pres[mesh.constraint_elements(*dims, "bottom-corners")] = 1
    pres[mesh.force_elements(*dims, "top-center")] = 1
    ro = oracle.simp(*dims, F, fixed, preserved=pres, max_iter=12, solver=1, penal_start=-1.0, continuation_iters=-1,
                     use_projection=1, beta_max=64.0, beta_interval=5, cg_tol=-1.0, cg_max_iter=400, stop_on_change=1,
                     volfrac=0.3, rmin=1.5)
    from topologyoptimization_b200 import TopologyOptimizerWorker3D
    w = TopologyOptimizerWorker3D()
    try:
        r = w.optimize({"nx": dims[0], "ny": dims[1], "nz": dims[2]},
                       dict(volumeFraction=0.3, maxIterations=12, penaltyFactor=3.0, filterRadius=1.5,
                            constraintPosition="bottom-corners", forceDirection="top-center", linearSolver="mgpcg"))
    finally:
        w.close()
    assert r["iterations"] == ro["iterations"]
    dc = np.abs(r["complianceHistory"] / ro["compliance"] - 1)
    dx = np.abs(r["densities"] - ro["x"]).max()
    print(f"corner supports: compliance rel max {dc.max():.3e}, x max abs {dx:.3e}, cg {list(r['cgIterations'])} vs "
          f"{list(ro['cg'])}")
    assert np.array_equal(r["cgIterations"], ro["cg"])
    assert dc.max() < 1e-10
    assert dx < 1e-6
