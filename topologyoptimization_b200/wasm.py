"""The reference's WASM solver exports (assembly/index.ts), served by libtpo.

Same names, argument meaning and return values as the WebAssembly functions, with
arrays in place of byte offsets into linear memory and no workspace pointer (the
library owns its scratch):

  applyAEbe3D(KEflat, edofs, E_vals, active, activeCount, p, Ap, ndof)   :403-439
  denseMatVecRaw(K, p, Ap, n)                                             :450-464
  ebePCG(dens, KEflat, edofs, F, U, freedofs, nel, edofSize, ndof, nfree,
         Emin, E0, penal, maxIter, tol) -> iterations                     :504-733
  ebeMGPCG(nelx, nely, nelz, dens, penal, F, U, fixedMask, maxIter, tol,
           KEflat=None, E0=1, Emin=1e-9) -> iterations                    :1076-1193
  ebeKSP_BDDC(nelx, nely, nelz, dens, penal, F, U, fixedMask, maxIter, tol,
              smootherIters=3, ...) -> iterations                         :1385-1517

ebeMGPCG takes the grid instead of the reference's 80-byte level descriptors: the
hierarchy (MGPrecond3D.ensure/updateFromFine, js/optimizer-worker-3d.js:408-582) is
built on the device by libtpo.  Outputs are written into the caller's arrays, as the
WASM functions write into linear memory.
"""
import numpy as np

from . import _native as N
from .problem import Problem


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def applyAEbe3D(KEflat, edofs, E_vals, active, activeCount, p, Ap, ndof):
    Ke, ed, ev, act, pv = _f64(KEflat), _i32(edofs), _f64(E_vals), _i32(active), _f64(p)
    out = np.empty(int(ndof))
    N.check(N.lib().tpo_apply_a_ebe3d(N.ptr(Ke), N.ptr(ed), N.ptr(ev), N.ptr(act), int(activeCount), len(ev),
                                      N.ptr(pv), N.ptr(out), int(ndof)), "applyAEbe3D")
    Ap[:int(ndof)] = out
    return None


def denseMatVecRaw(K, p, Ap, n):
    Kv, pv = _f64(K), _f64(p)
    out = np.empty(int(n))
    N.check(N.lib().tpo_dense_matvec(N.ptr(Kv), N.ptr(pv), N.ptr(out), int(n)), "denseMatVecRaw")
    Ap[:int(n)] = out
    return None


def ebePCG(dens, KEflat, edofs, F, U, freedofs, nel, edofSize, ndof, nfree, Emin, E0, penal, maxIter, tol):
    import ctypes as C
    d, Ke, ed, Fv, fr = _f64(dens), _f64(KEflat), _i32(edofs), _f64(F), _i32(freedofs)
    Uv = np.array(U[:int(ndof)], dtype=np.float64, copy=True)
    it = C.c_int32(0)
    st = N.lib().tpo_ebe_pcg(N.ptr(d), N.ptr(Ke), N.ptr(ed), N.ptr(Fv), N.ptr(Uv), N.ptr(fr), int(nel),
                             int(edofSize), int(ndof), int(nfree), float(Emin), float(E0), float(penal),
                             int(maxIter), float(tol), C.byref(it))
    N.check(st, "ebePCG", allow=(N.TPO_OK, N.TPO_NOT_CONVERGED))
    U[:int(ndof)] = Uv
    return it.value


def ebeMGPCG(nelx, nely, nelz, dens, penal, F, U, fixedMask, maxIter, tol, KEflat=None, E0=1.0, Emin=1e-9,
             nu=0.3, mg=None):
    with Problem(nelx, nely, nelz, fixedMask, Ke=KEflat, nu=nu, mg=mg) as P:
        P.set_densities(np.asarray(dens, dtype=np.float32), penal, E0, Emin)
        P.set_load(F)
        Uv, info = P.solve(None, precond=N.PREC_MG, max_iter=int(maxIter), tol=float(tol), warm_start=0,
                           ref_epsilon=1)
    U[:len(Uv)] = Uv
    return info.iterations


def ebeKSP_BDDC(nelx, nely, nelz, dens, penal, F, U, fixedMask, maxIter, tol, smootherIters=3, KEflat=None,
                E0=1.0, Emin=1e-9, nu=0.3):
    """ebeKSP_BDDC (assembly/index.ts:1385-1404) through tpo_ksp_bddc: the subdomain and
    corner descriptors the worker writes (KSPSolver._buildSubdomains,
    js/optimizer-worker-3d.js:1141-1231) are built on the device from the grid.  Returns
    the iteration count, as the WASM call."""
    import ctypes as C
    with Problem(nelx, nely, nelz, fixedMask, Ke=KEflat, nu=nu) as P:
        P.set_densities(np.asarray(dens, dtype=np.float32), penal, E0, Emin)
        Uv = np.zeros(P.ndof)
        it = C.c_int32(0)
        st = N.lib().tpo_ksp_bddc(P.h, N.ptr(np.ascontiguousarray(F, dtype=np.float64)), N.ptr(Uv), int(maxIter),
                                  float(tol), int(smootherIters), C.byref(it))
        N.check(st, "ebeKSP_BDDC", allow=(N.TPO_OK, N.TPO_NOT_CONVERGED))
    U[:len(Uv)] = Uv
    return it.value
