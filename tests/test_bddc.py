"""The reference's KSP CG with its "BDDC" preconditioner (ebeKSP_BDDC / bddcApply,
assembly/index.ts:1204-1517; subdomains of KSPSolver._buildSubdomains,
js/optimizer-worker-3d.js:1141-1231), the worker's linearSolver 'petsc' path.

The preconditioner averages subdomain-local Jacobi steps, adds undamped global Jacobi
sweeps and a Jacobi correction on the subdomain corners.  For the hex8 element matrix the
undamped sweeps amplify the upper spectrum of D^-1 K (lambda_max ~ 5.3), so the
preconditioner is indefinite and CG with it does not reduce the residual; the reference's
own test accepts that ("a weak preconditioner; verify it produces a finite residual",
tests/test-wasm-ksp-bddc.js:578-587).  The iteration is nevertheless stable to rounding
(a relative perturbation of 2^-52 in F moves U by ~1e-14 after 500 iterations), so the
device run is compared with the oracle's iterate by iterate: same iteration count, U
within 1e-9 relative after the same number of iterations."""
import numpy as np
import pytest

from conftest import cantilever_load, rel_inf


def _problem(oracle, dims):
    """setupProblem3D of the reference test (:121-147): x = 0 face fixed, -1 in y at the
    centre node of the x = nelx face."""
    nelx, nely, nelz = dims
    fixed = oracle.fixed_mask(*dims, "left")
    F = np.zeros(oracle.ndof_of(*dims))
    n = nelx * (nely + 1) * (nelz + 1) + (nely // 2) * (nelz + 1) + nelz // 2
    F[3 * n + 1] = -1.0
    return fixed, F


def test_oracle_partition_matches_worker_formula(oracle):
    """KSPSolver._buildSubdomains: ~8-64 subdomains, at least 2 per axis, never more than
    the elements along an axis except for the minimum of 2."""
    assert oracle.bddc_partition(4, 4, 4) == (2, 2, 2)
    assert oracle.bddc_partition(30, 10, 10) == (4, 2, 2)
    nsx, nsy, nsz = oracle.bddc_partition(256, 128, 128)
    assert 8 <= nsx * nsy * nsz <= 64 * 8 and min(nsx, nsy, nsz) >= 2
    assert oracle.bddc_partition(1, 5, 5)[0] == 2


def test_oracle_reference_scenarios(oracle):
    """tests/test-wasm-ksp-bddc.js Tests 2, 4, 5 on 4x4x4 solid (tol 1e-6, 500 iterations):
    a valid iteration count, a finite residual, a nonzero right face and zero fixed DOFs."""
    dims = (4, 4, 4)
    fixed, F = _problem(oracle, dims)
    U, it = oracle.ksp_bddc(*dims, oracle.lk(0.3), np.ones(64, np.float32), 3.0, fixed, F, 500, 1e-6)
    assert 0 < it <= 500
    mg = oracle.MG(*dims, oracle.lk(0.3), fixed)
    mg.update(np.ones(64, np.float32), 3.0)
    r = (F - mg.apply(U)) * (fixed == 0)
    assert np.isfinite(np.linalg.norm(r))
    right = [3 * (4 * 25 + j) + d for j in range(25) for d in range(3)]
    assert np.abs(U[right]).max() > 1e-10
    assert np.abs(U[fixed == 1]).max() < 1e-15


@pytest.mark.gpu
@pytest.mark.parametrize("dims,field", [((4, 4, 4), "solid"), ((8, 4, 4), "random"), ((12, 6, 6), "random"),
                                        ((21, 11, 9), "random"), ((2, 2, 2), "solid")])
@pytest.mark.parametrize("max_iter", [50, 500])
def test_bddc_iterates_match_oracle(native, oracle, dims, field, max_iter):
    from topologyoptimization_b200 import Problem
    nel = int(np.prod(dims))
    x = np.ones(nel, np.float32) if field == "solid" else np.random.default_rng(70).uniform(0.2, 1.0, nel).astype(
        np.float32)
    fixed, F = _problem(oracle, dims)
    Uo, ito = oracle.ksp_bddc(*dims, oracle.lk(0.3), x, 3.0, fixed, F, max_iter, 1e-6)
    with Problem(*dims, fixed) as P:
        P.set_densities(x, 3.0)
        P.set_load(F)
        U, info = P.solve(None, precond=native.PREC_BDDC, max_iter=max_iter, tol=1e-6, warm_start=0, ref_epsilon=1,
                          bddc_smoother_iters=3)
    assert info.iterations == ito
    assert np.isfinite(U).all() and not np.any(U[fixed == 1])
    assert rel_inf(U, Uo) < 1e-9


@pytest.mark.gpu
def test_bddc_worker_path(native, oracle):
    """linearSolver 'petsc' in the worker mirror runs the KSP/BDDC solve inside the SIMP
    loop: 6 iterations on 12x6x6 (penal 3, no projection, the worker's tolerance schedule,
    the cap min(nfree, 400)) against the oracle's loop with the same solver.  Every solve
    runs to the cap (the preconditioner is indefinite), so the compliance swings from step
    to step.  One such solve agrees with the oracle's to ~1e-12 (test above), but the loop
    feeds each step's float-rounded design into a solve that is far from converged, and
    from the fifth step on that amplifies the last-bit differences of the designs (measured
    on a B200: 1.6% at step 5).  Asserted: the same CG counts, the first four compliances
    within 1e-9 relative, and a finite run."""
    from topologyoptimization_b200 import TopologyOptimizerWorker3D
    dims = (12, 6, 6)
    fixed = oracle.fixed_mask(*dims, "left")
    F = np.zeros(oracle.ndof_of(*dims), np.float32)
    for j in range(dims[1] + 1):
        nn = dims[0] * (dims[1] + 1) * (dims[2] + 1) + j * (dims[2] + 1)
        F[3 * nn + 2] = -1.0
    pres = np.zeros(int(np.prod(dims)), np.uint8)
    pres[oracle.constraint_elements(*dims, "left")] = 1
    ro = oracle.simp(*dims, F, fixed, preserved=pres, max_iter=6, solver=4, penal_start=3.0, use_projection=0,
                     cg_tol=-1.0, cg_max_iter=400, stop_on_change=1, volfrac=0.3, rmin=1.5)
    w = TopologyOptimizerWorker3D()
    try:
        r = w.optimize({"nx": dims[0], "ny": dims[1], "nz": dims[2]},
                       dict(volumeFraction=0.3, maxIterations=6, penaltyFactor=3.0, filterRadius=1.5, penalStart=3.0,
                            useProjection=False, constraintPosition="left", F=F, preservedElements=pres.astype(bool),
                            linearSolver="petsc"))
    finally:
        w.close()
    assert r["iterations"] == ro["iterations"] == 6
    assert np.array_equal(r["cgIterations"], ro["cg"])
    dc = np.abs(r["complianceHistory"] / ro["compliance"] - 1)
    print(f"bddc worker: compliance rel, first four {dc[:4].max():.3e}, all {dc.max():.3e}")
    assert dc[:4].max() < 1e-9
    assert np.isfinite(r["complianceHistory"]).all() and np.isfinite(r["densities"]).all()


@pytest.mark.gpu
def test_ksp_bddc_export(native, oracle):
    """tpo_ksp_bddc (the ebeKSP_BDDC export, wasm.ebeKSP_BDDC) on the reference test's
    4x4x4 and an 8x4x4 random block: the oracle's iteration count and U within 1e-9."""
    from topologyoptimization_b200 import wasm
    for dims, seed in (((4, 4, 4), None), ((8, 4, 4), 71)):
        nel = int(np.prod(dims))
        x = np.ones(nel, np.float32) if seed is None else np.random.default_rng(seed).uniform(0.2, 1.0, nel).astype(
            np.float32)
        fixed, F = _problem(oracle, dims)
        Uo, ito = oracle.ksp_bddc(*dims, oracle.lk(0.3), x, 3.0, fixed, F, 200, 1e-6)
        U = np.zeros(len(F))
        it = wasm.ebeKSP_BDDC(*dims, x, 3.0, F, U, fixed, 200, 1e-6, smootherIters=3)
        assert it == ito
        assert rel_inf(U, Uo) < 1e-9
