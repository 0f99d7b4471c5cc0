"""Batched block MG-PCG (tpo_solve_multi_dev): nrhs load cases solved by one set of
kernels (right-hand side = grid z), each with its own PCG scalars.  Every right-hand side
runs the arithmetic of a single solve, so the batch reproduces the sequential solves."""
import numpy as np
import pytest

from conftest import rel_inf

pytestmark = pytest.mark.gpu


def point_loads(nelx, nely, nelz, nrhs, seed0=30):
    """Unit point loads at top-face nodes (z = nelz): position and direction from
    numpy.random.default_rng(seed0 + k), direction normalize(N(0, I3))."""
    from topologyoptimization_b200 import mesh
    F = np.zeros((nrhs, mesh.ndof(nelx, nely, nelz)))
    for k in range(nrhs):
        rng = np.random.default_rng(seed0 + k)
        ix, iy = int(rng.integers(0, nelx + 1)), int(rng.integers(0, nely + 1))
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        n = mesh.node_id(ix, iy, nelz, nely, nelz)
        F[k, 3 * n:3 * n + 3] = d
    return F


def _batched_vs_sequential(dims, bc, precision, tol, nrhs=8, max_iter=4000):
    import torch
    from topologyoptimization_b200 import Problem, mesh
    from topologyoptimization_b200 import _native as N
    x = np.random.default_rng(3).uniform(0.1, 1.0, int(np.prod(dims))).astype(np.float32)
    fixed = mesh.fixed_mask(*dims, bc)
    F = point_loads(*dims, nrhs)
    prec = N.FP64 if precision == "fp64" else N.F32_PRECOND
    opts = N.default_solve_opts(precond=N.PREC_MG, precision=prec, max_iter=max_iter, tol=tol, warm_start=0,
                                ref_epsilon=0)
    with Problem(*dims, fixed, mg=N.default_mg_opts(coarse_direct=1, safe_omega=1)) as P:
        P.set_densities(x, 3.0)
        dF = torch.from_numpy(F).cuda()
        dU = torch.zeros_like(dF)
        infos = P.solve_multi_dev(dF, dU, opts)
        Ub = dU.cpu().numpy()
        seq = []
        for k in range(nrhs):
            P.set_load(F[k])
            du = torch.zeros(F.shape[1], dtype=torch.float64, device="cuda")
            info = P.solve_dev(du, opts)
            seq.append((du.cpu().numpy(), info))
    summary = [(infos[k].iterations, seq[k][1].iterations, infos[k].converged, seq[k][1].converged,
                infos[k].rel_residual, seq[k][1].rel_residual) for k in range(nrhs)]
    for k in range(nrhs):
        Us, inf = seq[k]
        assert infos[k].iterations == inf.iterations, summary
        assert infos[k].converged == inf.converged, summary
        assert rel_inf(Ub[k], Us) < 1e-12, (k, rel_inf(Ub[k], Us), summary)
        assert abs(infos[k].compliance - F[k] @ Us) <= 1e-10 * abs(F[k] @ Us), summary
    return infos


@pytest.mark.parametrize("precision", ["fp64", "f32_precond"])
def test_batched_matches_sequential_bottom_corners(native, precision):
    """The batched load-case configuration's supports: the four corners of the z = 0 face."""
    _batched_vs_sequential((20, 10, 10), "bottom-corners", precision, 1e-8)


@pytest.mark.parametrize("precision", ["fp64", "f32_precond"])
def test_batched_matches_sequential_and_converges(native, precision):
    infos = _batched_vs_sequential((24, 12, 12), "left", precision, 1e-9, nrhs=5)
    assert all(i.converged == 1 and i.rel_residual < 1e-9 for i in infos)


def test_batched_warm_start_and_single_rhs_after(native):
    """A batch restarted from its own solution (warm start: the tolerance is relative to
    the restarted residual, as in the reference's FE solve) stays at that solution; a
    single solve on the same problem afterwards still works (the batch buffers are
    swapped back)."""
    import torch
    from topologyoptimization_b200 import Problem, mesh
    from topologyoptimization_b200 import _native as N
    dims, nrhs = (16, 8, 8), 4
    x = np.random.default_rng(7).uniform(0.2, 1.0, int(np.prod(dims))).astype(np.float32)
    fixed = mesh.fixed_mask(*dims, "left")
    F = point_loads(*dims, nrhs)
    with Problem(*dims, fixed, mg=N.default_mg_opts(coarse_direct=1, safe_omega=1)) as P:
        P.set_densities(x, 3.0)
        dF = torch.from_numpy(F).cuda()
        dU = torch.zeros_like(dF)
        opts = N.default_solve_opts(precond=N.PREC_MG, max_iter=3000, tol=1e-9, warm_start=0, ref_epsilon=0)
        first = P.solve_multi_dev(dF, dU, opts)
        assert all(i.converged == 1 for i in first)
        U0 = dU.cpu().numpy()
        opts.warm_start = 1
        infos = P.solve_multi_dev(dF, dU, opts)
        assert all(i.converged == 1 for i in infos)
        assert rel_inf(dU.cpu().numpy(), U0) < 1e-8
        P.set_load(F[1])
        U1, info = P.solve(None, opts=N.default_solve_opts(precond=N.PREC_MG, max_iter=3000, tol=1e-9, warm_start=0,
                                                            ref_epsilon=0))
        assert info.converged == 1
        assert rel_inf(U1, dU[1].cpu().numpy()) < 1e-6


def test_batched_rhs_pinned_to_oracle(native, oracle):
    """Each right-hand side of an 8-load-case batch at 20x10x10 (the batched configuration's
    corner supports and seeded top-face point loads, scaled by 1e6 so the reference's
    absolute shifts stay below the tolerance) solved as one block MG-PCG with the
    reference's hierarchy and recurrence, converged at 1e-12, against the oracle's
    ebeMGPCG of that load case alone: U within 1e-10 relative."""
    import torch
    from topologyoptimization_b200 import Problem, mesh
    from topologyoptimization_b200 import _native as N
    dims, nrhs = (20, 10, 10), 8
    x = np.random.default_rng(3).uniform(0.2, 1.0, int(np.prod(dims))).astype(np.float32)
    fixed = mesh.fixed_mask(*dims, "bottom-corners")
    F = point_loads(*dims, nrhs) * 1e6
    mg = oracle.MG(*dims, oracle.lk(0.3), fixed)
    mg.update(x, 3.0)
    with Problem(*dims, fixed) as P:
        P.set_densities(x, 3.0)
        dF = torch.from_numpy(F).cuda()
        dU = torch.zeros_like(dF)
        opts = N.default_solve_opts(precond=N.PREC_MG, max_iter=2000, tol=1e-12, warm_start=0, ref_epsilon=1)
        infos = P.solve_multi_dev(dF, dU, opts)
        Ub = dU.cpu().numpy()
    for k in range(nrhs):
        Uo, ito = mg.mgpcg(F[k], 2000, 1e-12)
        assert infos[k].converged == 1 and ito < 2000
        assert rel_inf(Ub[k], Uo) < 1e-10, (k, rel_inf(Ub[k], Uo))
