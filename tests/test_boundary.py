"""Entry points of the drop-in boundary beyond the solver: the GPUCompute energy seam,
the handle-based ebeMGPCG, the density-filter transpose and the host-array forward /
backward pair, each through the C ABI against the oracle or its device-array twin."""
import ctypes as C

import numpy as np
import pytest

from conftest import cantilever_load, rel_inf

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [(3, 2, 2), (16, 8, 8)])
def test_element_energies_match_wgsl_kernel(native, oracle, dims):
    """GPUCompute.computeElementEnergies (js/gpu-compute.js:187-303): float32 products and
    sums in the WGSL kernel's order, negative indices skipped; bit for bit against the
    oracle's restatement of that kernel."""
    from topologyoptimization_b200 import GPUCompute, mesh
    nel = int(np.prod(dims))
    rng = np.random.default_rng(60)
    U = rng.standard_normal(mesh.ndof(*dims)).astype(np.float32)
    KE = oracle.lk(0.3).astype(np.float32)
    ed = mesh.edofs3d(*dims).copy()
    ed[rng.random(ed.size) < 0.05] = -1
    g = GPUCompute()
    with pytest.raises(RuntimeError, match="GPU compute not available"):
        g.computeElementEnergies(U, KE, ed, nel, 24)
    assert g.init()
    got = g.computeElementEnergies(U, KE, ed, nel, 24)
    assert got.dtype == np.float32
    assert np.array_equal(got, oracle.element_energies_f32(U, KE, ed, nel, 24))


def test_mgpcg_export(native, oracle):
    """tpo_mgpcg: ebeMGPCG on a handle (cold start, the reference's recurrence) against the
    oracle's ebeMGPCG, converged at 1e-12."""
    from topologyoptimization_b200 import Problem
    from topologyoptimization_b200 import _native as N
    dims = (16, 8, 8)
    x = np.random.default_rng(61).uniform(0.2, 1.0, 1024).astype(np.float32)
    fixed = oracle.fixed_mask(*dims, "left")
    F = cantilever_load(*dims) * 1e6
    mg = oracle.MG(*dims, oracle.lk(0.3), fixed)
    mg.update(x, 3.0)
    Uo, ito = mg.mgpcg(F, 2000, 1e-12)
    with Problem(*dims, fixed) as P:
        P.set_densities(x, 3.0)
        U = np.zeros(len(F))
        it = C.c_int32()
        st = N.lib().tpo_mgpcg(P.h, N.ptr(np.ascontiguousarray(F)), N.ptr(U), 2000, 1e-12, C.byref(it))
    assert st == N.TPO_OK and it.value < 2000
    assert rel_inf(U, Uo) < 1e-10


@pytest.mark.parametrize("radius", [1.5, 4.5])
def test_density_filter_transpose(native, oracle, radius):
    """tpo_density_filter_transpose_dev is the transpose of the density filter H x / Hs of
    assembly/index.ts:224-273: against the dense matrix of the oracle's filter (a tiled
    stencil and, at radius 4.5, the per-element one)."""
    import torch
    from topologyoptimization_b200 import Problem, mesh
    dims = (7, 5, 4) if radius < 2 else (11, 10, 10)
    nel = int(np.prod(dims))
    H = np.stack([oracle.density_filter(np.eye(nel)[j], *dims, radius) for j in range(nel)], axis=1)
    g = np.random.default_rng(62).standard_normal(nel)
    with Problem(*dims, mesh.fixed_mask(*dims, "left")) as P:
        out = torch.empty(nel, dtype=torch.float64, device="cuda")
        P.density_filter_T_dev(radius, torch.from_numpy(g).cuda(), out)
        got = out.cpu().numpy()
    assert rel_inf(got, H.T @ g) < 1e-13


@pytest.mark.parametrize("with_l", [False, True])
def test_forward_backward_host_arrays(native, with_l):
    """tpo_forward / tpo_backward (host arrays, for bindings without device memory) give the
    objective and gradient of tpo_forward_dev / tpo_backward_dev bit for bit."""
    import torch
    from topologyoptimization_b200 import Problem, mesh
    from topologyoptimization_b200 import _native as N
    dims = (12, 6, 6)
    nel = int(np.prod(dims))
    rng = np.random.default_rng(63)
    x = rng.uniform(0.2, 0.8, nel)
    fixed = mesh.fixed_mask(*dims, "left")
    F = cantilever_load(*dims)
    l = rng.standard_normal(len(F)) * (fixed == 0) if with_l else None
    design = N.DesignOpts(penal=3.0, E0=1.0, Emin=1e-9, filter_radius=1.5)
    o = N.default_solve_opts(precond=N.PREC_MG, max_iter=2000, tol=1e-10, warm_start=0, ref_epsilon=0)
    with Problem(*dims, fixed) as P:
        P.set_load(F)
        J1, _ = P.forward_dev(torch.from_numpy(x).cuda(), design, o, d_l=None if l is None else torch.from_numpy(l).cuda())
        g1 = torch.empty(nel, dtype=torch.float64, device="cuda")
        P.backward_dev(g1, o, d_l=None if l is None else torch.from_numpy(l).cuda())
        g1 = g1.cpu().numpy()
        J2 = C.c_double()
        info = N.SolveInfo()
        st = N.lib().tpo_forward(P.h, C.byref(design), C.byref(o), N.ptr(x), N.ptr(l), C.byref(J2), C.byref(info))
        assert st == N.TPO_OK
        g2 = np.empty(nel)
        st = N.lib().tpo_backward(P.h, C.byref(o), N.ptr(l), N.ptr(g2), C.byref(info))
        assert st == N.TPO_OK
    assert J2.value == J1
    assert np.array_equal(g2, g1)


def test_volumetric_snapshot(native, oracle):
    """The stress snapshot of a SIMP step (_buildVolumetricSnapshot, js/optimizer-worker-3d.js:
    1579-1593, field of :2175-2184): stiffness x energy per element as float and its
    maximum, against the oracle's restatement on the step's own displacement field; the
    worker mirror returns it on stop and with every iteration on request."""
    import torch
    from topologyoptimization_b200 import Problem, TopologyOptimizerWorker3D, mesh
    from topologyoptimization_b200 import _native as N
    dims = (12, 6, 6)
    nel = int(np.prod(dims))
    x = np.random.default_rng(64).uniform(0.1, 1.0, nel).astype(np.float32)
    fixed = mesh.fixed_mask(*dims, "left")
    with Problem(*dims, fixed) as P:
        P.set_load(cantilever_load(*dims))
        with pytest.raises(N.TpoError):
            P.volumetric_snapshot()
        so = N.default_solve_opts(precond=N.PREC_MG, max_iter=500, tol=1e-10, warm_start=0, ref_epsilon=0)
        P.simp_step_dev(torch.from_numpy(x.copy()).cuda(),
                        N.SimpOpts(volfrac=0.3, penal=3.0, rmin=1.5, E0=1.0, Emin=1e-9, beta=1.0, use_projection=0,
                                   solve=so))
        stress, mx = P.volumetric_snapshot()
        energy = oracle.element_energy(oracle.lk(0.3), *dims, P.get_u())
    ref, mref = oracle.stress(x, energy, 3.0)
    assert rel_inf(stress, ref) < 1e-6
    assert abs(mx - mref) <= 1e-6 * mref
    w = TopologyOptimizerWorker3D()
    msgs = []
    try:
        r = w.optimize({"nx": 12, "ny": 6, "nz": 6},
                       dict(volumeFraction=0.3, maxIterations=2, penaltyFactor=3.0, filterRadius=1.5,
                            useProjection=False, F=cantilever_load(*dims), volumetricOutputMode="every-iteration"),
                       on_message=msgs.append)
    finally:
        w.close()
    vols = [m["volumetricData"] for m in msgs if m["type"] == "progress"]
    assert len(vols) == 2 and vols[1]["iteration"] == 2 and vols[1]["stress"].shape == (nel,)
    assert r["volumetricData"]["maxStress"] == vols[1]["maxStress"] > 0


@pytest.mark.gpu
def test_simp_step_host_arrays(native):
    """tpo_simp_step (the design and masks in host memory, copied in and back inside the
    call) gives the device-array step's design, compliance and change bit for bit over
    three SIMP iterations."""
    import torch
    from topologyoptimization_b200 import Problem, mesh
    from topologyoptimization_b200 import _native as N
    dims = (16, 8, 8)
    nel = int(np.prod(dims))
    fixed = mesh.fixed_mask(*dims, "left")
    F = cantilever_load(*dims)
    pres = np.zeros(nel, np.uint8)
    pres[mesh.constraint_elements(*dims, "left")] = 1
    x0 = np.full(nel, 0.3, np.float32)
    x0[pres == 1] = 1.0
    so = N.default_solve_opts(precond=N.PREC_MG, max_iter=500, tol=1e-8, warm_start=0, ref_epsilon=0)
    opts = N.SimpOpts(volfrac=0.3, penal=3.0, rmin=1.5, E0=1.0, Emin=1e-9, beta=1.0, use_projection=0, solve=so)
    hist = []
    for host in (True, False):
        with Problem(*dims, fixed) as P:
            P.set_load(F)
            x = x0.copy()
            d_x, d_p = torch.from_numpy(x0.copy()).cuda(), torch.from_numpy(pres).cuda()
            run = []
            for _ in range(3):
                info = P.simp_step(x, opts, pres) if host else P.simp_step_dev(d_x, opts, d_p)
                run.append((info.compliance, info.change, info.cg_iterations))
            hist.append((run, x if host else d_x.cpu().numpy()))
    assert hist[0][0] == hist[1][0]
    assert np.array_equal(hist[0][1], hist[1][1])
