"""GPUFEASolver: the reference's GPU solver class (js/gpu-fea-solver.js:73-845) on libtpo.

Same methods, argument meaning and error messages:
  init() -> bool                       (:91-141, async in the reference)
  isAvailable() -> bool                (:144-146)
  setup(params)                        (:162-191) raises 'GPUFEASolver: GPU not available'
  solve(options) -> {U, iterations, converged}
                                       (:704-820) raises 'GPUFEASolver: not initialized.
                                        Call init() and setup() first.'
  destroy()                            (:836-845)

The reference runs an FP32 Jacobi-PCG on WebGPU.  Here the solve is FP64 on the B200
(Jacobi-PCG by default, as the reference; ``solver='mgpcg'`` selects the multigrid
preconditioner) and U is returned as float32 unless ``returnF64`` is set.  When
``edofArray`` is the reference's structured numbering the grid is recovered from it
and the structured kernels are used; any other connectivity goes through the
general element-list path (tpo_ebe_pcg).
"""
import numpy as np

from . import _native as N
from . import mesh
from .problem import Problem


class GPUFEASolver:
    def __init__(self):
        self.available = False
        self._initialized = False
        self._problem = None
        self._key = None
        self._general = None
        self._setup_done = False
        self._nel = 0
        self._ndof = 0

    def init(self):
        if not self._initialized:
            self._initialized = True
            try:
                self.available = N.device_available()
            except ImportError:
                self.available = False
        return self.available

    def isAvailable(self):
        return bool(self.available)

    def setup(self, params):
        if not self.isAvailable():
            raise RuntimeError("GPUFEASolver: GPU not available")
        p = dict(params)
        nel, ndof = int(p["nel"]), int(p["ndof"])
        KE = np.asarray(p["KEflat"], dtype=np.float64)
        edofs = np.asarray(p["edofArray"], dtype=np.int32)
        dens = np.asarray(p["densities"], dtype=np.float32)
        F = np.asarray(p["F"], dtype=np.float64)
        fixed = np.asarray(p["fixedMask"], dtype=np.uint8)
        E0, Emin, penal = float(p["E0"]), float(p["Emin"]), float(p["penal"])
        self._solver = p.get("solver", "pcg")
        self._return_f64 = bool(p.get("returnF64", False))
        dims = None
        if all(k in p for k in ("nelx", "nely", "nelz")):
            dims = (int(p["nelx"]), int(p["nely"]), int(p["nelz"]))
        else:
            dims = mesh.structured_dims(edofs, nel, ndof)
        self._nel, self._ndof = nel, ndof
        if dims is not None:
            key = (dims, fixed.tobytes(), KE.tobytes())
            if self._problem is None or self._key != key:
                if self._problem is not None:
                    self._problem.close()
                self._problem = Problem(*dims, fixed, Ke=KE)
                self._key = key
            self._problem.set_densities(dens, penal, E0, Emin)
            self._problem.set_load(F)
            self._general = None
        else:
            if self._problem is not None:
                self._problem.close()
                self._problem = None
            self._general = dict(KE=KE, edofs=edofs, dens=dens.astype(np.float64), F=F,
                                 free=np.flatnonzero(fixed == 0).astype(np.int32), E0=E0, Emin=Emin, penal=penal)
        self._setup_done = True

    def solve(self, options=None):
        if not self.isAvailable() or not self._setup_done:
            raise RuntimeError("GPUFEASolver: not initialized. Call init() and setup() first.")
        o = options or {}
        max_it = int(o.get("maxIterations", 400))
        tol = float(o.get("tolerance", 1e-8))
        warm = o.get("warmStart")
        U0 = np.zeros(self._ndof) if warm is None else np.asarray(warm, dtype=np.float64)
        if self._problem is not None:
            prec = N.PREC_MG if self._solver == "mgpcg" else N.PREC_JACOBI
            U, info = self._problem.solve(U0, precond=prec, max_iter=max_it, tol=tol, warm_start=1, ref_epsilon=1)
            its, conv = int(info.iterations), bool(info.converged)
        else:
            from .wasm import ebePCG
            g = self._general
            U = U0.copy()
            its = ebePCG(g["dens"], g["KE"], g["edofs"], g["F"], U, g["free"], self._nel, 24, self._ndof,
                         len(g["free"]), g["Emin"], g["E0"], g["penal"], max_it, tol)
            conv = its < min(max_it, len(g["free"]))
        return {"U": U if self._return_f64 else U.astype(np.float32), "iterations": its, "converged": conv}

    def destroy(self):
        if self._problem is not None:
            self._problem.close()
        self._problem = None
        self._general = None
        self._setup_done = False
        self.available = False
        self._initialized = False
