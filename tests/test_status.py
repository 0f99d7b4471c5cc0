"""Error statuses of the C ABI on the GPU, each failure made on the host (a NaN in the
input, an iteration cap of 1, device memory already held by the caller, a bisection
cap): no kernel is made to fault, and the library stays usable after each."""
import ctypes as C

import numpy as np
import pytest

from conftest import cantilever_load

pytestmark = pytest.mark.gpu


def _solve_status(P, F, **kw):
    from topologyoptimization_b200 import _native as N
    P.set_load(F)
    o = N.default_solve_opts(**kw)
    U = np.zeros(P.ndof)
    info = N.SolveInfo()
    st = N.lib().tpo_solve(P.h, C.byref(o), N.ptr(U), C.byref(info))
    return st, info, U


@pytest.mark.parametrize("precond", ["jacobi", "mg"])
def test_nan_load_is_nonfinite(native, precond):
    from topologyoptimization_b200 import Problem, mesh
    dims = (8, 4, 4)
    fixed = mesh.fixed_mask(*dims, "left")
    F = cantilever_load(*dims)
    with Problem(*dims, fixed) as P:
        P.set_densities(np.full(128, 0.5, np.float32), 3.0)
        bad = F.copy()
        bad[np.flatnonzero(fixed == 0)[7]] = np.nan
        pc = native.PREC_MG if precond == "mg" else native.PREC_JACOBI
        st, _, _ = _solve_status(P, bad, precond=pc, max_iter=200, tol=1e-8)
        assert st == native.TPO_NONFINITE, native.status_string(st)
        st, info, _ = _solve_status(P, F, precond=pc, max_iter=2000, tol=1e-8)
        assert st == native.TPO_OK and info.converged == 1


def test_nan_load_ebe_pcg(native, oracle):
    from topologyoptimization_b200 import _native as N
    dims = (4, 3, 3)
    fixed = oracle.fixed_mask(*dims, "left")
    free = np.flatnonzero(fixed == 0).astype(np.int32)
    F = cantilever_load(*dims)
    F[free[3]] = np.nan
    U = np.zeros(len(F))
    it = C.c_int32()
    st = N.lib().tpo_ebe_pcg(N.ptr(np.ones(36)), N.ptr(oracle.lk(0.3)), N.ptr(oracle.edofs3d(*dims)), N.ptr(F),
                             N.ptr(U), N.ptr(free), 36, 24, len(F), len(free), 1e-9, 1.0, 3.0, 100, 1e-8, C.byref(it))
    assert st == N.TPO_NONFINITE


def test_iteration_cap_is_not_converged(native):
    from topologyoptimization_b200 import Problem, mesh
    dims = (8, 4, 4)
    fixed = mesh.fixed_mask(*dims, "left")
    with Problem(*dims, fixed) as P:
        P.set_densities(np.full(128, 0.5, np.float32), 3.0)
        for pc in (native.PREC_JACOBI, native.PREC_MG):
            st, info, U = _solve_status(P, cantilever_load(*dims), precond=pc, max_iter=1, tol=1e-8)
            assert st == native.TPO_NOT_CONVERGED and info.converged == 0 and info.iterations == 1
            assert np.isfinite(U).all() and np.any(U)  # the iterate is still written


def test_device_memory_exhausted_is_oom(native):
    """The caller holds all but 256 MB of the device; creating a 12.8M-DOF problem (whose
    hierarchy needs several GB) returns TPO_OOM and frees what it had taken, and the same
    creation succeeds once the memory is released."""
    import torch
    from topologyoptimization_b200 import Problem, mesh
    from topologyoptimization_b200 import _native as N
    dims = (256, 128, 128)
    fixed = mesh.fixed_mask(*dims, "left")
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info()
    hold = torch.empty(max(free - (256 << 20), 0), dtype=torch.uint8, device="cuda")
    try:
        with pytest.raises(N.TpoError) as e:
            Problem(*dims, fixed)
        assert e.value.status == N.TPO_OOM
    finally:
        del hold
        torch.cuda.empty_cache()
    with Problem(*dims, fixed) as P:
        assert P.levels >= 2


def test_bisection_cap_is_timeout(native):
    """An OC bisection cap below the steps the bracket needs returns TPO_TIMEOUT; the same
    call with the default cap succeeds."""
    import torch
    from topologyoptimization_b200 import Problem, mesh
    from topologyoptimization_b200 import _native as N
    dims = (8, 4, 4)
    rng = np.random.default_rng(3)
    x = torch.from_numpy(rng.uniform(0.1, 1, 128).astype(np.float32)).cuda()
    dc = torch.from_numpy((-rng.uniform(0.5, 2, 128) * 1e2).astype(np.float32)).cuda()
    xn = torch.empty_like(x)
    with Problem(*dims, mesh.fixed_mask(*dims, "left")) as P:
        with pytest.raises(N.TpoError) as e:
            P.oc_update_dev(x, dc, xn, 0.3, max_bisections=5)
        assert e.value.status == N.TPO_TIMEOUT
        ch, lm, nb = P.oc_update_dev(x, dc, xn, 0.3)
        assert nb > 5 and ch > 0
