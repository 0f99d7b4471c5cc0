"""B200 (sm_100a) implementation of the 3D SIMP finite-element path of
Jozo132/TopologyOptimization.

The product is libtpo.so (CUDA kernels + C ABI, include/tpo.h).  The Python modules
mirror the reference's interfaces on top of it:
  - GPUFEASolver                 js/gpu-fea-solver.js
  - GPUCompute                   js/gpu-compute.js (computeElementEnergies)
  - wasm.applyAEbe3D / ebePCG /
    denseMatVecRaw / ebeMGPCG    assembly/index.ts exports
  - TopologyOptimizerWorker3D    js/optimizer-worker-3d.js optimize()
  - worker2d.TopologyOptimizerWorker
                                 js/optimizer-worker.js optimize() (the 2D worker)
  - Problem                      device-resident handle (tpo_create ...)
"""
from .gpu_compute import GPUCompute  # noqa: F401
from .gpu_fea_solver import GPUFEASolver  # noqa: F401
from .problem import Problem, lk  # noqa: F401
from .worker3d import TopologyOptimizerWorker3D  # noqa: F401
from . import mesh, wasm, worker2d  # noqa: F401
