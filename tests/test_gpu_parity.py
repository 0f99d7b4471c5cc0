"""Parity of libtpo's CUDA path with the CPU oracle (oracle/tpo_oracle.c) on the same
seeded inputs.  Tolerances: bit-exact where the kernel follows the reference's
operation order (lk, general-edof apply, dense matvec, filters, OC given the same
sensitivities); 1e-12 relative (max norm) for the structured FP64 apply and one
V-cycle; 1e-10 relative for converged FP64 solves; float rounding (1 ulp class) for
float32-stored SIMP quantities."""
import os

import numpy as np
import pytest

from conftest import cantilever_load, rel_inf, top_center_load

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

GRIDS = [(1, 1, 1), (2, 2, 2), (5, 3, 7), (2, 9, 3), (16, 8, 8), (30, 10, 10), (13, 40, 5), (7, 3, 131)]


def _densities(nel, seed, lo=1e-3, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, nel).astype(np.float32)


def test_lk_bitwise(native, oracle):
    from topologyoptimization_b200 import lk
    for nu in (0.3, 0.25, 0.45):
        assert np.array_equal(lk(nu), oracle.lk(nu))


@pytest.mark.parametrize("dims", GRIDS)
def test_structured_apply(native, oracle, dims):
    from topologyoptimization_b200 import Problem, mesh
    nel = int(np.prod(dims))
    x = _densities(nel, 0)
    fixed = mesh.fixed_mask(*dims, "left")
    u = np.random.default_rng(1).standard_normal(mesh.ndof(*dims))
    Ke = oracle.lk(0.3)
    E = 1e-9 + x.astype(np.float64) ** 3 * (1 - 1e-9)
    act = np.flatnonzero(E > 1e-6).astype(np.int32)
    ref = oracle.apply_a(Ke, oracle.edofs3d(*dims), E, act, u)
    with Problem(*dims, fixed) as P:
        P.set_densities(x, 3.0)
        got = P.apply(u)
    assert rel_inf(got, ref) < 1e-12


def test_apply_golden(native):
    from topologyoptimization_b200 import Problem, mesh
    g = np.load(os.path.join(GOLDEN, "apply_5x3x4.npz"))
    with Problem(5, 3, 4, mesh.fixed_mask(5, 3, 4, "left")) as P:
        P.set_densities(g["x"], float(g["penal"]))
        assert rel_inf(P.apply(g["u"]), g["Ku"]) < 1e-12


def test_apply_f32(native, oracle):
    import torch
    from topologyoptimization_b200 import Problem, mesh
    dims = (16, 8, 8)
    nel = int(np.prod(dims))
    x = _densities(nel, 2)
    u = np.random.default_rng(3).standard_normal(mesh.ndof(*dims))
    with Problem(*dims, mesh.fixed_mask(*dims, "left")) as P:
        P.set_densities(x, 3.0)
        ref = P.apply(u)
        du = torch.from_numpy(u.astype(np.float32)).cuda()
        out = torch.empty_like(du)
        P.apply_f32_dev(du, out)
        torch.cuda.synchronize()
        assert rel_inf(out.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("ke_kind", ["synthetic", "hex8"])
@pytest.mark.parametrize("dims,frac", [((1, 1, 1), 1.0), ((3, 3, 3), 1.0), ((4, 4, 4), 0.5), ((6, 6, 6), 1.0)])
def test_wasm_apply_bitwise(native, oracle, ke_kind, dims, frac):
    """tests/test-wasm-applyA.js scenarios; the general-edof path matches bit for bit."""
    from topologyoptimization_b200 import wasm
    from test_oracle_pins import synthetic_ke
    rng = np.random.default_rng(11)
    nel = int(np.prod(dims))
    nd = oracle.ndof_of(*dims)
    Ke = synthetic_ke() if ke_kind == "synthetic" else oracle.lk(0.3)
    ed = oracle.edofs3d(*dims)
    E = rng.uniform(0.1, 1.0, nel)
    active = rng.permutation(nel)[: max(1, int(nel * frac))].astype(np.int32)
    p = rng.standard_normal(nd)
    Ap = np.empty(nd)
    wasm.applyAEbe3D(Ke, ed, E, active, len(active), p, Ap, nd)
    assert np.array_equal(Ap, oracle.apply_a(Ke, ed, E, active, p))
    wasm.applyAEbe3D(Ke, ed, E, active, len(active), np.zeros(nd), Ap, nd)
    assert not np.any(Ap)
    wasm.applyAEbe3D(Ke, ed, E, active, 0, p, Ap, nd)
    assert not np.any(Ap)


def test_dense_matvec_bitwise(native, oracle):
    from topologyoptimization_b200 import wasm
    rng = np.random.default_rng(3)
    K = rng.standard_normal((50, 50))
    p = rng.standard_normal(50)
    out = np.empty(50)
    wasm.denseMatVecRaw(K, p, out, 50)
    assert np.array_equal(out, oracle.dense_matvec(K, p))


@pytest.mark.parametrize("dims", [(8, 4, 4), (12, 6, 6), (5, 3, 7)])
def test_ebe_pcg(native, oracle, dims):
    from topologyoptimization_b200 import wasm
    nel = int(np.prod(dims))
    x = _densities(nel, 5, 0.2, 1.0).astype(np.float64)
    fixed = oracle.fixed_mask(*dims, "left")
    free = np.flatnonzero(fixed == 0).astype(np.int32)
    F = top_center_load(*dims) * 1e3
    Ke = oracle.lk(0.3)
    ed = oracle.edofs3d(*dims)
    nd = len(F)
    U0 = np.random.default_rng(6).standard_normal(nd) * 1e-3  # warm start
    Uo, ito = oracle.ebe_pcg(x, Ke, ed, F, U0, free, nd, 1e-9, 1.0, 3.0, 5000, 1e-10)
    Ug = U0.copy()
    itg = wasm.ebePCG(x, Ke, ed, F, Ug, free, nel, 24, nd, len(free), 1e-9, 1.0, 3.0, 5000, 1e-10)
    assert abs(itg - ito) <= 2
    assert rel_inf(Ug, Uo) < 1e-9
    # zero force, cold start: converged at 0 iterations with U = 0
    Uz = np.zeros(nd)
    assert wasm.ebePCG(x, Ke, ed, np.zeros(nd), Uz, free, nel, 24, nd, len(free), 1e-9, 1.0, 3.0, 100, 1e-8) == 0
    assert not np.any(Uz)


@pytest.mark.parametrize("dims,pos", [((8, 4, 4), "left"), ((30, 10, 10), "left"), ((16, 8, 8), "bottom-corners"),
                                      ((21, 11, 9), "left"), ((64, 32, 32), "left")])
def test_vcycle(native, oracle, dims, pos):
    from topologyoptimization_b200 import Problem
    nel = int(np.prod(dims))
    x = _densities(nel, 7, 0.05, 1.0)
    fixed = oracle.fixed_mask(*dims, pos)
    b = np.random.default_rng(8).standard_normal(len(fixed)) * (fixed == 0)
    mg = oracle.MG(*dims, oracle.lk(0.3), fixed)
    mg.update(x, 3.0)
    ref = mg.vcycle(b)
    with Problem(*dims, fixed) as P:
        assert P.levels == mg.num_levels
        P.set_densities(x, 3.0)
        got = P.vcycle(b)
    assert rel_inf(got, ref) < 1e-11


def _void_design(dims, seed=0):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    x = rng.uniform(0.2, 1.0, nx * ny * nz).astype(np.float32)
    x[rng.random(x.size) < 0.5] = 1e-3
    x.reshape(nz, ny, nx)[:, :, 0] = 1.0
    x.reshape(nz, ny, nx)[0, :, nx - 1] = 1.0  # the elements under the loaded line stay solid
    return x


@pytest.mark.parametrize("dims", [(8, 4, 4), (24, 12, 12), (32, 16, 16)])
@pytest.mark.parametrize("coarse_direct", [0, 1])
def test_vcycle_safe_omega(native, oracle, dims, coarse_direct):
    """Per-level damping (safe_omega): structured levels from the bound on Ke, dense levels
    from the device-side Gershgorin bound; same V-cycle as the oracle's."""
    from topologyoptimization_b200 import Problem
    from topologyoptimization_b200 import _native as N
    x = _void_design(dims)
    fixed = oracle.fixed_mask(*dims, "left")
    b = np.random.default_rng(8).standard_normal(len(fixed)) * (fixed == 0)
    mg = oracle.MG(*dims, oracle.lk(0.3), fixed, coarse_direct=coarse_direct, safe_omega=1)
    mg.update(x, 3.0)
    ref = mg.vcycle(b)
    with Problem(*dims, fixed, mg=N.default_mg_opts(coarse_direct=coarse_direct, safe_omega=1)) as P:
        P.set_densities(x, 3.0)
        got = P.vcycle(b)
    assert rel_inf(got, ref) < 1e-10
    assert b @ got > 0


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed_3xtf32", "f32_precond", "f32_precond_tc",
                                       "f32_precond_3xtf32", "f32_precond_bf16"])
def test_mgpcg_safe_omega_converges(native, oracle, precision):
    """On a half-void design the safe-damped MG-PCG reaches 1e-8 (true residual)."""
    from topologyoptimization_b200 import Problem
    from topologyoptimization_b200 import _native as N
    dims = (32, 16, 16)
    x = _void_design(dims, seed=3)
    fixed = oracle.fixed_mask(*dims, "left")
    F = cantilever_load(*dims)
    with Problem(*dims, fixed, mg=N.default_mg_opts(coarse_direct=1, safe_omega=1)) as P:
        P.set_load(F)
        P.set_densities(x, 3.0)
        kw = {"fp64": dict(precision=N.FP64), "mixed": dict(precision=N.MIXED, inner_tol=0.3),
              "f32_precond": dict(precision=N.F32_PRECOND),
              "mixed_3xtf32": dict(precision=N.MIXED, inner_tol=0.3, tensor_cores=4),
              "f32_precond_tc": dict(precision=N.F32_PRECOND, tensor_cores=1),
              "f32_precond_3xtf32": dict(precision=N.F32_PRECOND, tensor_cores=3),
              "f32_precond_bf16": dict(precision=N.F32_PRECOND, tensor_cores=5)}[precision]
        U, info = P.solve(opts=N.default_solve_opts(precond=N.PREC_MG, max_iter=2000, tol=1e-8, warm_start=0,
                                                     ref_epsilon=0, **kw))
        Ku = P.apply(U)
    r = (F - Ku) * (fixed == 0)
    assert info.converged == 1
    assert np.linalg.norm(r) < 1.01e-8 * np.linalg.norm(F * (fixed == 0))


@pytest.mark.parametrize("dims,pos,graded", [((4, 4, 4), "bottom-corners", False), ((6, 6, 6), "bottom-corners", False),
                                             ((4, 4, 4), "bottom-corners", True), ((30, 10, 10), "left", True),
                                             ((32, 16, 16), "left", True)])
def test_mgpcg(native, oracle, dims, pos, graded):
    from topologyoptimization_b200 import wasm
    nel = int(np.prod(dims))
    x = (0.3 + 0.7 * np.arange(nel) / nel) if graded else np.ones(nel)
    x = x.astype(np.float32)
    fixed = oracle.fixed_mask(*dims, pos)
    F = top_center_load(*dims) if pos == "bottom-corners" else cantilever_load(*dims)
    mg = oracle.MG(*dims, oracle.lk(0.3), fixed)
    mg.update(x, 3.0)
    Uo, ito = mg.mgpcg(F, 500, 1e-6)
    Ug = np.zeros_like(F)
    itg = wasm.ebeMGPCG(*dims, x, 3.0, F, Ug, fixed, 500, 1e-6)
    assert abs(itg - ito) <= 1
    assert rel_inf(Ug, Uo) < 1e-8
    assert abs(F @ Ug - F @ Uo) / abs(F @ Uo) < 1e-9


def test_mgpcg_golden(native):
    from topologyoptimization_b200 import wasm
    g = np.load(os.path.join(GOLDEN, "mgpcg_4x4x4_graded.npz"))
    U = np.zeros_like(g["F"])
    it = wasm.ebeMGPCG(4, 4, 4, g["x"], 3.0, g["F"], U, g["fixed"], int(g["max_iter"]), float(g["tol"]))
    assert abs(it - int(g["iters"])) <= 1
    assert rel_inf(U, g["U"]) < 1e-8


def test_mgpcg_zero_force(native):
    from topologyoptimization_b200 import mesh, wasm
    fixed = mesh.fixed_mask(4, 4, 4, "bottom-corners")
    U = np.ones(mesh.ndof(4, 4, 4))
    it = wasm.ebeMGPCG(4, 4, 4, np.ones(64, np.float32), 3.0, np.zeros_like(U), U, fixed, 500, 1e-6)
    assert it == 0 and not np.any(U)


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("dims", [(5, 3, 7), (16, 8, 8), (30, 10, 10)])
def test_simp_pieces(native, oracle, dims):
    import torch
    from topologyoptimization_b200 import Problem, mesh
    nel = int(np.prod(dims))
    rng = np.random.default_rng(9)
    x = rng.uniform(0.05, 1.0, nel).astype(np.float32)
    U = rng.standard_normal(mesh.ndof(*dims))
    Ke = oracle.lk(0.3)
    with Problem(*dims, mesh.fixed_mask(*dims, "left")) as P:
        en = torch.empty(nel, dtype=torch.float32, device="cuda")
        P.element_energy_dev(_dev(U), en)
        en_ref = oracle.element_energy(Ke, *dims, U)
        assert rel_inf(en.cpu().numpy(), en_ref) < 1e-6
        xp = torch.empty_like(en)
        P.heaviside_dev(_dev(x), 8.0, xp)
        xp_ref = oracle.heaviside(x, 8.0)
        assert np.abs(xp.cpu().numpy() - xp_ref).max() < 2e-7
        dc = torch.empty_like(en)
        P.sensitivity_dev(_dev(x), _dev(xp_ref), _dev(en_ref), 3.0, 1.0, 8.0, True, dc)
        dc_ref = oracle.sensitivity(x, xp_ref, en_ref, 3.0, 1.0, 8.0, True)
        assert rel_inf(dc.cpu().numpy(), dc_ref) < 1e-6
        for rmin in (1.5, 2.0, 2.7, 4.9, 5.5):  # tiled kernels up to a half-width of 4, then per element
            dcn = torch.empty_like(en)
            P.filter_sens_dev(rmin, _dev(x), _dev(dc_ref), dcn)
            hs = oracle.filter_hs(*dims, rmin)
            assert np.array_equal(dcn.cpu().numpy(), oracle.filter_sens(*dims, rmin, hs, x, dc_ref))
        d64 = torch.empty(nel, dtype=torch.float64, device="cuda")
        for radius in (1.5, 2.0, 4.0, 4.5):
            P.density_filter_dev(radius, _dev(x.astype(np.float64)), d64)
            assert np.array_equal(d64.cpu().numpy(), oracle.density_filter(x.astype(np.float64), *dims, radius))
        xnew = torch.empty_like(en)
        lm, nb = P.oc_dev(_dev(x), 0.3, _dev(-np.abs(dc_ref)), xnew)
        xr, lmr, nbr = oracle.oc(x, 0.3, -np.abs(dc_ref))
        assert nb == nbr and lm == lmr
        assert np.array_equal(xnew.cpu().numpy(), xr)


def test_simp_loop_matches_oracle(native, oracle):
    """8 SIMP iterations (12x4x4 cantilever, MGPCG at fixed tol 1e-8): compliance
    history and final densities against the oracle's run."""
    from topologyoptimization_b200 import TopologyOptimizerWorker3D
    g = np.load(os.path.join(GOLDEN, "simp_12x4x4.npz"))
    w = TopologyOptimizerWorker3D()
    cfg = dict(volumeFraction=0.3, maxIterations=8, penaltyFactor=3.0, filterRadius=1.5, penalStart=3.0,
               useProjection=False, constraintPosition="left", F=g["F"], cgTolerance=1e-8, linearSolver="mgpcg",
               preservedElements=g["preserved"].astype(bool))
    r = w.optimize({"nx": 12, "ny": 4, "nz": 4}, cfg)
    w.close()
    assert r["iterations"] == len(g["compliance"])
    assert np.abs(r["complianceHistory"] / g["compliance"] - 1).max() < 1e-6
    assert np.abs(r["densities"] - g["x"]).max() < 1e-4


def test_gpu_fea_solver_api(native, oracle):
    from topologyoptimization_b200 import GPUFEASolver, mesh
    dims = (8, 4, 4)
    nel = int(np.prod(dims))
    s = GPUFEASolver()
    with pytest.raises(RuntimeError, match="not initialized"):
        s.solve({})
    assert s.init() and s.isAvailable()
    x = _densities(nel, 12, 0.2, 1.0)
    fixed = mesh.fixed_mask(*dims, "left")
    F = top_center_load(*dims).astype(np.float32) * 1e3
    s.setup(dict(KEflat=oracle.lk(0.3).astype(np.float32), edofArray=mesh.edofs3d(*dims), densities=x, F=F,
                 fixedMask=fixed, nel=nel, ndof=len(F), E0=1.0, Emin=1e-9, penal=3.0))
    r = s.solve({"maxIterations": 2000, "tolerance": 1e-10})
    assert r["U"].dtype == np.float32 and r["converged"] and r["iterations"] > 0
    free = np.flatnonzero(fixed == 0).astype(np.int32)
    Uo, _ = oracle.ebe_pcg(x.astype(np.float64), oracle.lk(0.3).astype(np.float32).astype(np.float64),
                           oracle.edofs3d(*dims), F.astype(np.float64), np.zeros(len(F)), free, len(F), 1e-9, 1.0,
                           3.0, 5000, 1e-10)
    assert rel_inf(r["U"], Uo) < 1e-6
    s.destroy()
    assert not s.isAvailable()


@pytest.mark.parametrize("dims", [(32, 16, 16), (48, 24, 24)])
def test_mixed_precision_solve(native, oracle, dims):
    """FP32 MGPCG with FP64 reliable updates reaches the FP64 tolerance on the true
    residual; its compliance and U agree with the FP64 MGPCG solution."""
    from topologyoptimization_b200 import Problem, mesh
    nel = int(np.prod(dims))
    x = _densities(nel, 21, 0.05, 1.0)
    fixed = mesh.fixed_mask(*dims, "left")
    F = cantilever_load(*dims)
    with Problem(*dims, fixed) as P:
        P.set_densities(x, 3.0)
        P.set_load(F)
        U64, i64 = P.solve(None, precond=native.PREC_MG, max_iter=2000, tol=1e-10, warm_start=0, ref_epsilon=0)
        Um, im = P.solve(None, precond=native.PREC_MG, precision=native.MIXED, max_iter=2000, tol=1e-10,
                         warm_start=0, ref_epsilon=0, inner_tol=0.1)
    assert i64.converged and im.converged and im.outer_iterations >= 2
    assert im.iterations <= 2 * i64.iterations + 5  # the Krylov space survives the updates
    assert im.rel_residual < 1e-10
    assert abs(im.compliance - i64.compliance) / abs(i64.compliance) < 1e-9
    assert rel_inf(Um, U64) < 1e-7


@pytest.mark.parametrize("dims", [(5, 3, 7), (16, 8, 8), (30, 10, 10), (13, 40, 37)])
def test_apply_tf32_tensor_cores(native, oracle, dims):
    """tcgen05 TF32 element contraction against the FP64 apply: TF32 operands carry a
    10-bit mantissa, so the max-norm relative error stays at the 1e-3 level."""
    import torch
    from topologyoptimization_b200 import Problem, mesh
    nel = int(np.prod(dims))
    x = _densities(nel, 4)
    u = np.random.default_rng(5).standard_normal(mesh.ndof(*dims))
    with Problem(*dims, mesh.fixed_mask(*dims, "left")) as P:
        P.set_densities(x, 3.0)
        ref = P.apply(u)
        du = torch.from_numpy(u.astype(np.float32)).cuda()
        out = torch.zeros_like(du)
        P.apply_tf32_dev(du, out)
        torch.cuda.synchronize()
        assert rel_inf(out.cpu().numpy(), ref) < 5e-3


@pytest.mark.parametrize("dims", [(5, 3, 7), (16, 8, 8), (30, 10, 10), (13, 40, 37), (64, 33, 70)])
def test_apply_3xtf32_tensor_cores(native, oracle, dims):
    """3xTF32 element contraction (Ke and E_e u_e split into TF32 high and low parts):
    FP32-class accuracy against the FP64 apply, far below plain TF32's error."""
    import torch
    from topologyoptimization_b200 import Problem, mesh
    nel = int(np.prod(dims))
    x = _densities(nel, 4)
    u = np.random.default_rng(5).standard_normal(mesh.ndof(*dims))
    with Problem(*dims, mesh.fixed_mask(*dims, "left")) as P:
        P.set_densities(x, 3.0)
        ref = P.apply(u.astype(np.float32).astype(np.float64))
        du = torch.from_numpy(u.astype(np.float32)).cuda()
        o3, o1, o32 = torch.zeros_like(du), torch.zeros_like(du), torch.zeros_like(du)
        P.apply_3xtf32_dev(du, o3)
        P.apply_tf32_dev(du, o1)
        P.apply_f32_dev(du, o32)
        torch.cuda.synchronize()
        e3 = rel_inf(o3.cpu().numpy(), ref)
        e1 = rel_inf(o1.cpu().numpy(), ref)
        e32 = rel_inf(o32.cpu().numpy(), ref)
    assert e3 < 2e-5 and e32 < 2e-5
    assert e3 < 0.05 * e1


@pytest.mark.parametrize("dims", [(5, 3, 7), (16, 8, 8), (30, 10, 10), (13, 40, 37)])
def test_apply_bf16_tensor_cores(native, oracle, dims):
    """BF16 tcgen05 element contraction (kind::f16, K padded to 32) against the FP64 apply:
    the 8-bit mantissa of the operands bounds the max-norm relative error near 1e-2."""
    import torch
    from topologyoptimization_b200 import Problem, mesh
    nel = int(np.prod(dims))
    x = _densities(nel, 4)
    u = np.random.default_rng(5).standard_normal(mesh.ndof(*dims))
    with Problem(*dims, mesh.fixed_mask(*dims, "left")) as P:
        P.set_densities(x, 3.0)
        ref = P.apply(u)
        du = torch.from_numpy(u.astype(np.float32)).cuda()
        ob, ot = torch.zeros_like(du), torch.zeros_like(du)
        P.apply_bf16_dev(du, ob)
        P.apply_tf32_dev(du, ot)
        torch.cuda.synchronize()
        eb = rel_inf(ob.cpu().numpy(), ref)
        et = rel_inf(ot.cpu().numpy(), ref)
    assert eb < 5e-2 and eb > et


def test_mixed_precision_tensor_cores(native):
    """The mixed-precision solve with TF32 tensor-core applies in the fine-level smoother
    and residual still reaches the FP64 tolerance on the true residual."""
    from topologyoptimization_b200 import Problem, mesh
    dims = (32, 16, 16)
    nel = int(np.prod(dims))
    x = _densities(nel, 21, 0.05, 1.0)
    F = cantilever_load(*dims)
    with Problem(*dims, mesh.fixed_mask(*dims, "left")) as P:
        P.set_densities(x, 3.0)
        P.set_load(F)
        U64, i64 = P.solve(None, precond=native.PREC_MG, max_iter=2000, tol=1e-10, warm_start=0, ref_epsilon=0)
        Ut, it = P.solve(None, precond=native.PREC_MG, precision=native.MIXED, max_iter=3000, tol=1e-10,
                         warm_start=0, ref_epsilon=0, inner_tol=0.1, tensor_cores=1)
    
    assert it.converged and it.rel_residual < 1e-10
    assert abs(it.compliance - i64.compliance) / abs(i64.compliance) < 1e-9
    assert rel_inf(Ut, U64) < 1e-7


@pytest.mark.parametrize("dims", [(16, 8, 8), (32, 16, 16)])
def test_vcycle_coarse_direct(native, oracle, dims):
    """V-cycle whose coarsest (dense Galerkin) level is solved directly: the GPU inverts
    the coarse operator once per density update, the oracle runs a Cholesky solve."""
    from topologyoptimization_b200 import Problem
    nel = int(np.prod(dims))
    x = _densities(nel, 17, 0.05, 1.0)
    fixed = oracle.fixed_mask(*dims, "left")
    b = np.random.default_rng(18).standard_normal(len(fixed)) * (fixed == 0)
    mg = oracle.MG(*dims, oracle.lk(0.3), fixed, coarse_direct=1)
    mg.update(x, 3.0)
    ref = mg.vcycle(b)
    with Problem(*dims, fixed, mg=native.default_mg_opts(coarse_direct=1)) as P:
        P.set_densities(x, 3.0)
        got = P.vcycle(b)
    assert rel_inf(got, ref) < 1e-9


def _chebyshev_coefficients(Ke, ratio, m):
    """Chebyshev iteration on [kappa / ratio, kappa], kappa = lambda_max(diag(Ke)^-1 Ke):
    sweep 0 weight 1 / theta, sweep k >= 1 (cd_k, cr_k) (Adams et al. 2003)."""
    K = Ke.reshape(24, 24)
    kappa = np.linalg.eigvals(K / np.diag(K)[:, None]).real.max()
    lmax, lmin = kappa, kappa / ratio
    theta, delta = 0.5 * (lmax + lmin), 0.5 * (lmax - lmin)
    sigma = theta / delta
    rho, coef = 1.0 / sigma, [(0.0, 1.0 / theta)]
    for _ in range(1, m):
        rn = 1.0 / (2.0 * sigma - rho)
        coef.append((rn * rho, 2.0 * rn / delta))
        rho = rn
    return coef


@pytest.mark.parametrize("coarse_iters", [3, 20])
def test_chebyshev_smoother_matches_recurrence(native, oracle, coarse_iters):
    """Chebyshev smoothing (mg option chebyshev): on a one-level hierarchy the V-cycle is
    one smoothing sequence from zero, x_{k+1} = x_k + cd_k (x_k - x_{k-1}) + cr_k D^-1
    (b - K x_k) on free DOFs; the same recurrence in numpy on the oracle's K u, for a
    short sequence and one of 22 sweeps (each sweep its own coefficients)."""
    from topologyoptimization_b200 import Problem
    dims = (8, 4, 6)
    nel = int(np.prod(dims))
    x = _densities(nel, 41, 0.05, 1.0)
    fixed = oracle.fixed_mask(*dims, "left")
    b = np.random.default_rng(42).standard_normal(len(fixed)) * (fixed == 0)
    Ke = oracle.lk(0.3)
    edofs = oracle.edofs3d(*dims)
    E = 1e-9 + x.astype(np.float64) ** 3 * (1 - 1e-9)
    act = np.flatnonzero(E > 1e-6).astype(np.int32)
    D = np.zeros(len(fixed))
    dk = np.diag(Ke.reshape(24, 24))
    ed = np.asarray(edofs).reshape(-1, 24)
    for e in act:
        np.add.at(D, ed[e], E[e] * dk)
    invD = np.where((fixed == 0) & (D > 0), 1.0 / np.where(D > 0, D, 1.0), 0.0)
    nu1, ratio = 2, 16.0
    coef = _chebyshev_coefficients(Ke, ratio, nu1 + coarse_iters)
    xk, xprev = np.zeros(len(fixed)), np.zeros(len(fixed))
    for cd, cr in coef:
        r = b - oracle.apply_a(Ke, edofs, E, act, xk)
        xn = xk + cd * (xk - xprev) + cr * invD * r
        xn[fixed != 0] = xk[fixed != 0]
        xprev, xk = xk, xn
    mg = native.default_mg_opts(max_levels=1, nu1=nu1, coarse_iters=coarse_iters, safe_omega=1, chebyshev=1,
                                cheb_ratio=ratio)
    with Problem(*dims, fixed, mg=mg) as P:
        P.set_densities(x, 3.0)
        got = P.vcycle(b)
    assert rel_inf(got, xk) < 1e-12


def test_chebyshev_vcycle_symmetric_and_converges(native, oracle):
    """The Chebyshev V-cycle is symmetric positive definite (the same polynomial before
    and after the coarse correction) and its MG-PCG reaches 1e-8 on a half-void design, in
    FP64, with the FP32 preconditioner and with the FP32 preconditioner whose fine-level
    Chebyshev sweeps run on the TF32 tensor-core apply, in no more FP64 iterations than
    damped Jacobi."""
    from topologyoptimization_b200 import Problem
    from topologyoptimization_b200 import _native as N
    dims = (32, 16, 16)
    x = _void_design(dims, seed=5)
    fixed = oracle.fixed_mask(*dims, "left")
    F = cantilever_load(*dims)
    rng = np.random.default_rng(6)
    iters = {}
    for cheb in (0, 1):
        with Problem(*dims, fixed, mg=N.default_mg_opts(coarse_direct=1, safe_omega=1, chebyshev=cheb)) as P:
            P.set_densities(x, 3.0)
            P.set_load(F)
            if cheb:
                b1 = rng.standard_normal(len(fixed)) * (fixed == 0)
                b2 = rng.standard_normal(len(fixed)) * (fixed == 0)
                v1, v2 = P.vcycle(b1), P.vcycle(b2)
                assert abs(b1 @ v2 - b2 @ v1) < 1e-10 * abs(b1 @ v2)
                assert b1 @ v1 > 0 and b2 @ v2 > 0
            for prec, tc in ((N.FP64, 0), (N.F32_PRECOND, 0), (N.F32_PRECOND, 1)):
                if tc and not cheb:
                    continue
                U, info = P.solve(opts=N.default_solve_opts(precond=N.PREC_MG, max_iter=2000, tol=1e-8, warm_start=0,
                                                             ref_epsilon=0, precision=prec, tensor_cores=tc))
                r = (F - P.apply(U)) * (fixed == 0)
                assert info.converged == 1
                assert np.linalg.norm(r) < 1.01e-8 * np.linalg.norm(F * (fixed == 0))
                iters[(cheb, prec, tc)] = info.iterations
    assert iters[(1, N.FP64, 0)] <= iters[(0, N.FP64, 0)], iters


@pytest.mark.parametrize("dims", [(4, 4, 4), (5, 4, 4), (16, 8, 8), (21, 11, 9)])
def test_galerkin_levels_bitwise(native, oracle, dims):
    """Dense Galerkin levels (_assembleGalerkinFromElements / _assembleGalerkinFromMatrix,
    js/optimizer-worker-3d.js:628-699) are the oracle's matrices bit for bit: the device
    gathers every coarse entry in the reference's summation order, with no atomics.  A
    rebuild and a second problem give the same bits, and so does the V-cycle."""
    from topologyoptimization_b200 import Problem
    nel = int(np.prod(dims))
    x = _densities(nel, 31, 0.05, 1.0)
    fixed = oracle.fixed_mask(*dims, "left")
    mg = oracle.MG(*dims, oracle.lk(0.3), fixed)
    mg.update(x, 3.0)
    b = np.random.default_rng(32).standard_normal(len(fixed)) * (fixed == 0)
    dense = 0
    with Problem(*dims, fixed) as P, Problem(*dims, fixed) as Q:
        P.set_densities(x, 3.0)
        Q.set_densities(x, 3.0)
        v1 = P.vcycle(b)
        for li in range(P.levels):
            if not P.level_info(li)["dense"]:
                continue
            dense += 1
            K = P.level_dense(li)
            Ko = mg.level_arrays(li)[2]
            assert np.array_equal(K, Ko), f"level {li}: max diff {np.abs(K - Ko).max():.3e}"
            assert np.array_equal(K, Q.level_dense(li))
        P.set_densities(x, 3.0)
        assert np.array_equal(P.vcycle(b), v1)
        assert np.array_equal(Q.vcycle(b), v1)
    assert dense >= 1


@pytest.mark.parametrize("n", [3000, 4194304])
@pytest.mark.parametrize("move", [0.2, 0.1])
def test_oc_update_exact_volume(native, oracle, n, move):
    """OC with the move limit and the change test (tpo_oc_update_dev, OC :3066-3101,
    :2244-2247): x_new bit for bit, lambda, the bisection count and the change against the
    oracle, up to 4,194,304 elements with denormal-range, tiny and zero densities mixed in.
    The device sums each step's volume exactly (as an integer in units of 2^-149) and
    rounds once, so its decisions do not depend on the launch shape."""
    import torch
    from topologyoptimization_b200 import Problem, mesh
    rng = np.random.default_rng(40)
    x = rng.uniform(0, 1, n).astype(np.float32)
    tiny = rng.random(n) < 0.01
    x[tiny] = (10.0 ** rng.uniform(-44, -8, int(tiny.sum()))).astype(np.float32)
    x[rng.random(n) < 0.01] = 0.0
    dc = (-rng.uniform(0.5, 2.0, n) * 1e2).astype(np.float32)
    dims = (256, 128, 128) if n == 4194304 else (30, 10, 10)
    xr, lmr, nbr = oracle.oc(x, 0.3, dc, move=move)
    with Problem(*dims, mesh.fixed_mask(*dims, "left")) as P:
        d_x, d_dc = _dev(x), _dev(dc)
        d_xn = torch.empty_like(d_x)
        ch, lm, nb = P.oc_update_dev(d_x, d_dc, d_xn, 0.3, move=move)
        xn = d_xn.cpu().numpy()
    assert nb == nbr and lm == lmr
    assert np.array_equal(xn, xr)
    assert ch == np.abs(xr.astype(np.float64) - x.astype(np.float64)).max()
