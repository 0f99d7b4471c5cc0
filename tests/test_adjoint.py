"""Differentiable forward/backward (tpo_forward_dev / tpo_backward_dev) and the grounded
spring: parity with the oracle, the compliance gradient against the reference's own
sensitivity formula (js/optimizer-worker-3d.js:2175-2192), and central finite
differences for a displacement objective with an output spring (the config of a
compliant mechanism: 96x48x48, x ~ U[0.2, 0.8], input force +1 in x at the centre of the
x = 96 face, output z-displacement with spring k = 0.01)."""
import numpy as np
import pytest

from conftest import rel_inf

pytestmark = pytest.mark.gpu


def _solve_opts(N, tol=1e-12):
    return N.default_solve_opts(precond=N.PREC_MG, precision=N.FP64, max_iter=5000, tol=tol, warm_start=0,
                                ref_epsilon=0)


def _setup(dims, seed_x=3, seed_out=4):
    from topologyoptimization_b200 import mesh
    nx, ny, nz = dims
    x = np.random.default_rng(seed_x).uniform(0.2, 0.8, nx * ny * nz)
    fixed = mesh.fixed_mask(nx, ny, nz, "left")
    F = np.zeros(mesh.ndof(nx, ny, nz))
    F[3 * mesh.node_id(nx, ny // 2, nz // 2, ny, nz) + 0] = 1.0
    rng = np.random.default_rng(seed_out)
    on = mesh.node_id(int(rng.integers(1, nx + 1)), int(rng.integers(0, ny + 1)), int(rng.integers(0, nz + 1)), ny, nz)
    out_dof = 3 * on + 2
    return x, fixed, F, out_dof


def _problem(dims, fixed, F, out_dof, k=0.01):
    from topologyoptimization_b200 import Problem
    from topologyoptimization_b200 import _native as N
    P = Problem(*dims, fixed, mg=N.default_mg_opts(coarse_direct=1, safe_omega=1))
    P.set_load(F)
    if out_dof is not None:
        P.set_spring(out_dof, k)
    return P


def test_spring_apply_and_vcycle_match_oracle(native, oracle):
    from topologyoptimization_b200 import _native as N
    dims = (12, 6, 6)
    x, fixed, F, out_dof = _setup(dims)
    x32 = x.astype(np.float32)
    b = np.random.default_rng(9).standard_normal(len(F)) * (fixed == 0)
    mg = oracle.MG(*dims, oracle.lk(0.3), fixed, coarse_direct=1, safe_omega=1)
    mg.set_spring(out_dof, 0.01)
    mg.update(x32, 3.0)
    with _problem(dims, fixed, F, out_dof) as P:
        P.set_densities(x32, 3.0)
        assert rel_inf(P.apply(b), mg.apply(b)) < 1e-12
        assert rel_inf(P.vcycle(b), mg.vcycle(b)) < 1e-10
        P.set_spring(-1, 0.0)
        assert rel_inf(P.apply(b), mg.apply(b)) > 1e-9  # the spring was really in the apply
        mg.set_spring(-1, 0.0)
        assert rel_inf(P.apply(b), mg.apply(b)) < 1e-12


def _fwd(P, x, design, N, l=None):
    import torch
    J, info = P.forward_dev(torch.from_numpy(x).cuda(), design, _solve_opts(N), d_l=l)
    assert info.converged == 1
    return J


def test_compliance_gradient_matches_reference_sensitivity(native, oracle):
    """For J = F.u the adjoint is u itself: dJ/dxPhys = -p xPhys^(p-1) (E0 - Emin) u_e^T Ke u_e.
    The reference's dc uses E0 and a float32 energy; they agree to float rounding."""
    import torch
    from topologyoptimization_b200 import adjoint
    from topologyoptimization_b200 import _native as N
    dims = (16, 8, 8)
    x, fixed, F, _ = _setup(dims)
    design = adjoint.design_opts(filter_radius=1.5)
    with _problem(dims, fixed, F, None) as P:
        J = _fwd(P, x, design, N)
        U = P.get_u()
        gphys = torch.empty(x.size, dtype=torch.float64, device="cuda")
        grad = torch.empty_like(gphys)
        P.backward_dev(grad, _solve_opts(N), d_grad_phys=gphys)
        gphys = gphys.cpu().numpy()
    assert abs(J - F @ U) < 1e-12 * abs(J)
    xphys = oracle.density_filter(x, *dims, 1.5)
    en = oracle.element_energy(oracle.lk(0.3), *dims, U)
    dc_ref = oracle.sensitivity(xphys.astype(np.float32), xphys.astype(np.float32), en, 3.0, 1.0, 1.0, False)
    assert rel_inf(gphys, dc_ref) < 1e-5


def test_displacement_gradient_central_differences(native):
    """J = u_z(out) with an output spring: adjoint gradient through SIMP and the density
    filter transpose against central differences (h = 1e-6, FP64 solves to 1e-12)."""
    import torch
    from topologyoptimization_b200 import adjoint
    from topologyoptimization_b200 import _native as N
    dims = (12, 6, 6)
    x, fixed, F, out_dof = _setup(dims)
    design = adjoint.design_opts(filter_radius=1.5)
    l = np.zeros(len(F))
    l[out_dof] = 1.0
    dl = torch.from_numpy(l).cuda()
    with _problem(dims, fixed, F, out_dof) as P:
        _fwd(P, x, design, N, dl)
        grad = torch.empty(x.size, dtype=torch.float64, device="cuda")
        info = P.backward_dev(grad, _solve_opts(N), d_l=dl)
        assert info.converged == 1
        grad = grad.cpu().numpy()
        elems = np.random.default_rng(5).choice(x.size, 24, replace=False)
        h = 1e-6
        fd = []
        for e in elems:
            xp, xm = x.copy(), x.copy()
            xp[e] += h
            xm[e] -= h
            fd.append((_fwd(P, xp, design, N, dl) - _fwd(P, xm, design, N, dl)) / (2 * h))
    fd = np.array(fd)
    assert np.linalg.norm(grad[elems] - fd) < 1e-5 * np.linalg.norm(fd)


def test_autograd_function(native):
    import torch
    from topologyoptimization_b200 import adjoint
    from topologyoptimization_b200 import _native as N
    dims = (12, 6, 6)
    x, fixed, F, _ = _setup(dims)
    design = adjoint.design_opts(filter_radius=1.5)
    with _problem(dims, fixed, F, None) as P:
        xt = torch.from_numpy(x).cuda().requires_grad_(True)
        J = adjoint.FEObjective().apply(xt, P, design, _solve_opts(N), None)
        (2.0 * J).backward()
        g = torch.empty(x.size, dtype=torch.float64, device="cuda")
        P.backward_dev(g, _solve_opts(N))
        assert rel_inf(xt.grad.cpu().numpy(), 2.0 * g.cpu().numpy()) < 1e-14


def test_mechanism_config_fd_64_elements(native):
    """The full compliant-mechanism configuration: 96x48x48 (698,691 DOF), FD on 64
    elements drawn with seed 5."""
    import torch
    from topologyoptimization_b200 import adjoint
    from topologyoptimization_b200 import _native as N
    dims = (96, 48, 48)
    x, fixed, F, out_dof = _setup(dims)
    design = adjoint.design_opts(filter_radius=1.5)
    l = np.zeros(len(F))
    l[out_dof] = 1.0
    dl = torch.from_numpy(l).cuda()
    with _problem(dims, fixed, F, out_dof) as P:
        _fwd(P, x, design, N, dl)
        grad = torch.empty(x.size, dtype=torch.float64, device="cuda")
        assert P.backward_dev(grad, _solve_opts(N), d_l=dl).converged == 1
        grad = grad.cpu().numpy()
        elems = np.random.default_rng(5).choice(x.size, 64, replace=False)
        h = 1e-6
        fd = np.array([(_fwd(P, np.where(np.arange(x.size) == e, x + h, x), design, N, dl)
                        - _fwd(P, np.where(np.arange(x.size) == e, x - h, x), design, N, dl)) / (2 * h)
                       for e in elems])
    assert np.linalg.norm(grad[elems] - fd) < 1e-4 * np.linalg.norm(fd)
