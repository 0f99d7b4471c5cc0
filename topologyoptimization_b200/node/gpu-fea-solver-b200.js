// Drop-in GPUFEASolver (js/gpu-fea-solver.js:73-845) and GPUCompute
// (js/gpu-compute.js:9-542, the method the worker calls) on libtpo through the N-API
// addon built from tpo_napi.cc.  Same class names, methods, arguments and error messages,
// so js/optimizer-worker-3d.js needs only its imports changed:
//   import { GPUFEASolver, GPUCompute } from './gpu-fea-solver-b200.js';
import { createRequire } from 'module';

const require = createRequire(import.meta.url);
const tpo = require('./build/Release/tpo_napi.node');

export class GPUFEASolver {
    constructor() {
        this.available = false;
        this._h = null;
        this._setup = false;
    }

    async init() {
        this.available = tpo.deviceAvailable();
        return this.available;
    }

    isAvailable() {
        return this.available;
    }

    // params: KEflat (Float32Array 576), edofArray (Int32Array), densities (Float32Array),
    // F (Float32Array), fixedMask (Uint8Array), nel, ndof, E0, Emin, penal; optional
    // solver: 'pcg' (the reference's Jacobi-PCG, default) or 'mgpcg'
    setup(params) {
        if (!this.isAvailable()) throw new Error('GPUFEASolver: GPU not available');
        this._h = tpo.setup(this._h, params);  // keeps the device problem while grid, Ke and supports are unchanged
        this._setup = true;
    }

    async solve({ maxIterations = 400, tolerance = 1e-8, warmStart = null } = {}) {
        if (!this.isAvailable() || !this._setup) {
            throw new Error('GPUFEASolver: not initialized. Call init() and setup() first.');
        }
        return tpo.solve(this._h, maxIterations, tolerance, warmStart);  // {U: Float32Array, iterations, converged}
    }

    // Extension: one whole iteration of the worker's SIMP loop (projection, solve, energies,
    // sensitivities, filter, OC, change) on the device problem of the last setup(); x
    // (Float32Array, nel) is updated in place.  options: volfrac, penal, rmin, beta,
    // useProjection, tolerance, maxIterations.  -> {compliance, change, cgIterations}
    simpStep(options, x, preserved = null, voidMask = null) {
        if (!this.isAvailable() || !this._setup) {
            throw new Error('GPUFEASolver: not initialized. Call init() and setup() first.');
        }
        return tpo.simpStep(this._h, options, x, preserved, voidMask);
    }

    destroy() {
        if (this._h) tpo.destroy(this._h);
        this._h = null;
        this._setup = false;
        this.available = false;
    }
}

export class GPUCompute {
    constructor() {
        this.available = false;
    }

    async init() {
        this.available = tpo.deviceAvailable();
        return this.available;
    }

    isAvailable() {
        return this.available;
    }

    async computeElementEnergies(U, KEflat, edofs, nel, edofSize) {
        if (!this.isAvailable()) throw new Error('GPU compute not available');
        return tpo.computeElementEnergies(U, KEflat, edofs, nel, edofSize);
    }

    destroy() {
        this.available = false;
    }
}

// The WASM export surface of assembly/index.ts, for the worker's wasmModule.exports
// calls (_solveWithWasmPCG :3572-3629): arrays instead of byte offsets, no workspace.
export const tpoExports = {
    ebePCG: (...args) => tpo.ebePCG(...args),
    applyAEbe3D: (...args) => tpo.applyAEbe3D(...args),
    denseMatVecRaw: (...args) => tpo.denseMatVecRaw(...args),
    // (nelx, nely, nelz, KEflat, densities, penal, E0, Emin, fixedMask, F, U, maxIter, tol,
    //  smootherIters): the subdomains are built from the grid, not passed as descriptors
    ebeKSP_BDDC: (...args) => tpo.ebeKSP_BDDC(...args),
};

// The chosen form's differentiable objective J = l.u (the compliance when l is null):
// forward() solves, backward() returns dJ/dx through SIMP and the density filter.
export class FEObjective {
    constructor(solver, design /* {penal, E0, Emin, filterRadius} */) {
        this.solver = solver;
        this.design = design;
        this.l = null;
    }

    async forward(x /* Float64Array(nel) */, l = null /* Float64Array(ndof) or null */) {
        this.l = l;
        return tpo.forward(this.solver._h, this.design, x, l);
    }

    async backward() {
        return tpo.backward(this.solver._h, this.l);  // Float64Array(nel)
    }
}
