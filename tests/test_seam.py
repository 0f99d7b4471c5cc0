"""The Node addon's call sequence for the GPUFEASolver seam (js/gpu-fea-solver.js:73-845),
topologyoptimization_b200/node/tpo_seam.h, compiled into a C++ harness and run against
libtpo: the same sequence the addon's setup() / solve() make, without a Node runtime.
Its results must equal the Python mirror's (same library calls) bit for bit and the
oracle's Jacobi-PCG at the drop-in bar."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, cantilever_load, rel_inf

HARNESS = os.path.join(ROOT, "tests", "harness", "seam_harness.cc")
LIBDIR = os.path.join(ROOT, "topologyoptimization_b200")


def build_harness(out_dir):
    exe = os.path.join(str(out_dir), "seam_harness")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-I",
                           os.path.join(LIBDIR, "node"), HARNESS, "-L", LIBDIR, "-ltpo", f"-Wl,-rpath,{LIBDIR}",
                           "-o", exe])
    return exe


def test_harness_and_seam_header_compile(tmp_path):
    """tpo_seam.h (the addon's call sequence) and the harness compile against include/tpo.h."""
    exe = build_harness(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


def _write_input(path, Ke32, edofs, dens, dens2, F32, fixed, solver_mg, maxit, tol, E0=1.0, Emin=1e-9, penal=3.0):
    nel, ndof = len(dens), len(F32)
    with open(path, "wb") as f:
        np.array([nel, ndof], np.int64).tofile(f)
        np.array([solver_mg, maxit], np.int32).tofile(f)
        np.array([E0, Emin, penal, tol], np.float64).tofile(f)
        np.ascontiguousarray(Ke32, np.float32).tofile(f)
        np.ascontiguousarray(edofs, np.int32).tofile(f)
        np.ascontiguousarray(dens, np.float32).tofile(f)
        np.ascontiguousarray(dens2, np.float32).tofile(f)
        np.ascontiguousarray(F32, np.float32).tofile(f)
        np.ascontiguousarray(fixed, np.uint8).tofile(f)


def _read_output(path, ndof):
    raw = open(path, "rb").read()
    out, off = [], 0
    for _ in range(2):
        st, it, conv = np.frombuffer(raw, np.int32, 3, off)
        off += 12
        U = np.frombuffer(raw, np.float32, ndof, off)
        off += 4 * ndof
        U64 = np.frombuffer(raw, np.float64, ndof, off)
        off += 8 * ndof
        out.append(dict(status=int(st), iterations=int(it), converged=int(conv), U=U, U64=U64))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["pcg", "mgpcg"])
@pytest.mark.parametrize("structured", [True, False])
def test_seam_sequence_on_gpu(native, oracle, tmp_path, solver, structured):
    from topologyoptimization_b200 import GPUFEASolver, mesh
    if solver == "mgpcg" and not structured:
        pytest.skip("the element-list path is Jacobi-PCG only")
    dims = (12, 6, 6)
    nel = int(np.prod(dims))
    rng = np.random.default_rng(50)
    x = rng.uniform(0.2, 1.0, nel).astype(np.float32)
    x2 = np.clip(x + rng.uniform(-0.1, 0.1, nel), 0.2, 1.0).astype(np.float32)
    fixed = mesh.fixed_mask(*dims, "left")
    F = (cantilever_load(*dims) * 1e6).astype(np.float32)
    Ke32 = oracle.lk(0.3).astype(np.float32)
    ed = mesh.edofs3d(*dims)
    if not structured:  # the same mesh with its elements listed in reverse: not the worker's numbering
        ed = ed.reshape(-1, 24)[::-1].ravel().copy()
        x, x2 = x[::-1].copy(), x2[::-1].copy()
    exe = build_harness(tmp_path)
    inp, outp = os.path.join(tmp_path, "in.bin"), os.path.join(tmp_path, "out.bin")
    maxit, tol = 5000, 1e-12
    _write_input(inp, Ke32, ed, x, x2, F, fixed, int(solver == "mgpcg"), maxit, tol)
    r = subprocess.run([exe, inp, outp], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    res = _read_output(outp, len(F))
    # the Python mirror makes the same library calls
    s = GPUFEASolver()
    assert s.init()
    params = dict(KEflat=Ke32, edofArray=ed, densities=x, F=F, fixedMask=fixed, nel=nel, ndof=len(F), E0=1.0,
                  Emin=1e-9, penal=3.0, solver=solver, returnF64=True)
    s.setup(params)
    r0 = s.solve({"maxIterations": maxit, "tolerance": tol})
    s.setup(dict(params, densities=x2))
    r1 = s.solve({"maxIterations": maxit, "tolerance": tol, "warmStart": res[0]["U"]})
    if structured:
        # the addon's simpStep (seam_simp_step -> tpo_simp_step): two SIMP iterations from
        # densities2 on the same problem, against the same library call made here
        from topologyoptimization_b200 import _native as N
        raw = open(outp, "rb").read()
        off = 2 * (12 + 12 * len(F))
        steps = []
        for _ in range(2):
            st, cg = np.frombuffer(raw, np.int32, 2, off)
            c, ch = np.frombuffer(raw, np.float64, 2, off + 8)
            steps.append((int(st), int(cg), float(c), float(ch)))
            off += 24
        xh = np.frombuffer(raw, np.float32, nel, off)
        so = N.default_solve_opts(precond=N.PREC_MG if solver == "mgpcg" else N.PREC_JACOBI, max_iter=maxit,
                                  tol=1e-8, warm_start=0 if solver == "mgpcg" else 1, ref_epsilon=1)
        opts = N.SimpOpts(volfrac=0.3, penal=3.0, rmin=1.5, E0=1.0, Emin=1e-9, beta=1.0, use_projection=0,
                          guard_sensitivities=0, solve=so)
        xp = x2.copy()
        for k in range(2):
            info = s._problem.simp_step(xp, opts)
            assert steps[k] == (0, info.cg_iterations, info.compliance, info.change)
        assert np.array_equal(xh, xp)
    s.destroy()
    for got, ref in ((res[0], r0), (res[1], r1)):
        assert got["status"] == 0 and got["converged"] == 1
        assert got["iterations"] == ref["iterations"]
        assert np.array_equal(got["U64"], ref["U"])
        assert np.array_equal(got["U"], got["U64"].astype(np.float32))
    # against the oracle's Jacobi-PCG / ebeMGPCG on the f32 element matrix the worker passes
    free = np.flatnonzero(fixed == 0).astype(np.int32)
    Ke64 = Ke32.astype(np.float64)
    if solver == "pcg":
        Uo, _ = oracle.ebe_pcg(x.astype(np.float64), Ke64, ed, F.astype(np.float64), np.zeros(len(F)), free, len(F),
                               1e-9, 1.0, 3.0, maxit, tol)
    else:
        mg = oracle.MG(*dims, Ke64, fixed)
        mg.update(x, 3.0)
        Uo, _ = mg.fe_pcg(F.astype(np.float64), np.zeros(len(F)), maxit, tol, precond="mg")
    assert rel_inf(res[0]["U64"], Uo) < 1e-10
