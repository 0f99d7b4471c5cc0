"""GPUCompute: the reference's WebGPU helper class (js/gpu-compute.js:9-542) on libtpo,
restricted to the method the SIMP worker calls on its hot path.

  init() -> bool                                         (:20-58, async in the reference)
  isAvailable() -> bool                                  (:60-70)
  computeElementEnergies(U, KEflat, edofs, nel, edofSize) -> float32[nel]
                                                         (:187-303; called by the worker
                                                          at js/optimizer-worker-3d.js:2146)
  destroy()                                              (:535-542)

The energies are those of the reference's WGSL kernel: float32 products and sums in its
loop order, negative DOF indices skipped (tpo_element_energies).  computeElementEnergies
raises 'GPU compute not available' before init(), as the reference throws.
"""
import numpy as np

from . import _native as N


class GPUCompute:
    def __init__(self):
        self.available = False
        self._initialized = False

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

    def computeElementEnergies(self, U, KEflat, edofs, nel, edofSize):
        if not self.isAvailable():
            raise RuntimeError("GPU compute not available")
        Uf = np.ascontiguousarray(U, dtype=np.float32)
        Kf = np.ascontiguousarray(KEflat, dtype=np.float32)
        ed = np.ascontiguousarray(edofs, dtype=np.int32)
        nel, es = int(nel), int(edofSize)
        if ed.size < nel * es or Kf.size < es * es:
            raise ValueError("edofs or KEflat shorter than nel * edofSize / edofSize^2")
        out = np.empty(nel, dtype=np.float32)
        N.check(N.lib().tpo_element_energies(N.ptr(Uf), N.ptr(Kf), N.ptr(ed), nel, es, Uf.size, N.ptr(out)),
                "computeElementEnergies")
        return out

    def destroy(self):
        self.available = False
        self._initialized = False
