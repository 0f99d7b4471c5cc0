// tpo_seam.h -- the call sequence the Node binding makes on libtpo for the reference's
// GPUFEASolver seam (js/gpu-fea-solver.js:73-845), as plain C++ over the C ABI of
// include/tpo.h.  The N-API addon (tpo_napi.cc) wraps these functions; the test harness
// (tests/harness/seam_harness.cc) calls them directly, so the sequence is exercised on a
// GPU even where no Node runtime exists.
//
//   seam_setup   GPUFEASolver.setup(params)                         (:162-191)
//   seam_solve   GPUFEASolver.solve({maxIterations, tolerance,
//                                    warmStart}) -> {U, iterations, converged}  (:704-820)
//   seam_destroy GPUFEASolver.destroy()                             (:836-845)
//   seam_simp_step one iteration of the worker's loop (js/optimizer-worker-3d.js:2074-2301)
//   seam_ksp_bddc wasmModule.exports.ebeKSP_BDDC (assembly/index.ts:1385-1404)
//
// setup receives what the worker passes (js/optimizer-worker-3d.js:4102-4125): KEflat
// (float32, 576), edofArray (int32, nel*24), densities (float32, nel), F (float32, ndof),
// fixedMask (uint8, ndof), nel, ndof, E0, Emin, penal.  The grid is recovered from the
// structured edofArray (the worker's numbering, js/optimizer-worker-3d.js:1448-1494);
// any other connectivity is solved through the element-list path (tpo_ebe_pcg).  The
// device problem is kept across setup calls with the same grid, Ke and fixed mask.
#pragma once
#include <stdint.h>

#include <cstring>
#include <string>
#include <vector>

#include "tpo.h"

namespace tpo_seam {

// The worker's element numbering e = ex + ey*nelx + ez*nelx*nely with the local node
// order (0,0,0),(1,0,0),(1,1,0),(0,1,0),(0,0,1),(1,0,1),(1,1,1),(0,1,1) and node
// n = x*nny*nnz + y*nnz + z.
inline void edofs3d(int nelx, int nely, int nelz, std::vector<int32_t> &ed) {
    const int nny = nely + 1, nnz = nelz + 1;
    static const int ox[8] = {0, 1, 1, 0, 0, 1, 1, 0}, oy[8] = {0, 0, 1, 1, 0, 0, 1, 1},
                     oz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    ed.resize((size_t)nelx * nely * nelz * 24);
    for (int ez = 0; ez < nelz; ez++)
        for (int ey = 0; ey < nely; ey++)
            for (int ex = 0; ex < nelx; ex++) {
                const size_t e = (size_t)ex + (size_t)ey * nelx + (size_t)ez * nelx * nely;
                for (int b = 0; b < 8; b++) {
                    const long long n = (long long)(ex + ox[b]) * nny * nnz + (long long)(ey + oy[b]) * nnz + (ez + oz[b]);
                    for (int c = 0; c < 3; c++) ed[e * 24 + 3 * b + c] = (int32_t)(3 * n + c);
                }
            }
}

// (nelx, nely, nelz) when edofs is the structured numbering of a grid with nel elements
// and ndof DOFs; false otherwise.
inline bool structured_dims(const int32_t *edofs, int64_t nel, int64_t ndof, int dims[3]) {
    if (!edofs || nel < 1 || edofs[0] != 0) return false;
    const long long nnz = edofs[9] / 3, nynz = edofs[3] / 3;
    if (nnz < 2 || nynz % nnz) return false;
    const long long nny = nynz / nnz;
    if (ndof % (3 * nynz)) return false;
    const long long nnx = ndof / (3 * nynz);
    const long long nx = nnx - 1, ny = nny - 1, nz = nnz - 1;
    if (nx < 1 || ny < 1 || nz < 1 || nx * ny * nz != nel) return false;
    std::vector<int32_t> ref;
    edofs3d((int)nx, (int)ny, (int)nz, ref);
    if (std::memcmp(ref.data(), edofs, ref.size() * sizeof(int32_t)) != 0) return false;
    dims[0] = (int)nx;
    dims[1] = (int)ny;
    dims[2] = (int)nz;
    return true;
}

struct SetupParams {
    const float *KEflat = nullptr;       // 576
    const int32_t *edofArray = nullptr;  // nel * 24
    const float *densities = nullptr;    // nel
    const float *F = nullptr;            // ndof
    const uint8_t *fixedMask = nullptr;  // ndof
    int64_t nel = 0, ndof = 0;
    double E0 = 1.0, Emin = 1e-9, penal = 3.0;
    int solver_mg = 0;  // opt-in field solver: 'mgpcg' (1) or 'pcg' (0, the reference's Jacobi-PCG)
};

struct State {
    tpo_problem *p = nullptr;
    int dims[3] = {0, 0, 0};
    std::vector<double> Ke64;
    std::vector<uint8_t> fixed;
    bool structured = false;
    bool ready = false;
    int solver_mg = 0;
    int64_t nel = 0, ndof = 0;
    // element-list path (non-structured connectivity)
    std::vector<double> dens64, F64;
    std::vector<int32_t> edofs, freedofs;
    double E0 = 1.0, Emin = 1e-9, penal = 3.0;
    std::string error;
};

inline tpo_status fail_with(State &s, tpo_status st) {
    const char *m = tpo_last_error();
    s.error = std::string(tpo_status_string(st)) + ": " + (m ? m : "");
    return st;
}

inline void seam_destroy(State &s) {
    if (s.p) tpo_destroy(s.p);
    s.p = nullptr;
    s.ready = false;
}

// GPUFEASolver.setup.  Returns TPO_NO_DEVICE when no GPU is usable (the reference throws
// 'GPUFEASolver: GPU not available').
inline tpo_status seam_setup(State &s, const SetupParams &q) {
    if (!tpo_device_available()) {
        s.error = "GPUFEASolver: GPU not available";
        return TPO_NO_DEVICE;
    }
    if (!q.KEflat || !q.edofArray || !q.densities || !q.F || !q.fixedMask || q.nel < 1 || q.ndof < 1) {
        s.error = "GPUFEASolver: invalid setup parameters";
        return TPO_BAD_ARG;
    }
    std::vector<double> Ke(q.KEflat, q.KEflat + 576);
    std::vector<uint8_t> fixed(q.fixedMask, q.fixedMask + q.ndof);
    int dims[3];
    const bool structured = structured_dims(q.edofArray, q.nel, q.ndof, dims);
    s.solver_mg = q.solver_mg;
    s.nel = q.nel;
    s.ndof = q.ndof;
    s.E0 = q.E0;
    s.Emin = q.Emin;
    s.penal = q.penal;
    tpo_status st = TPO_OK;
    if (structured) {
        const bool same = s.p && s.structured && std::memcmp(s.dims, dims, sizeof(dims)) == 0 && s.Ke64 == Ke &&
                          s.fixed == fixed;
        if (!same) {
            seam_destroy(s);
            tpo_mg_opts mg;
            tpo_default_mg_opts(&mg);
            const tpo_grid g{dims[0], dims[1], dims[2]};
            st = tpo_create(&g, Ke.data(), 0.3, fixed.data(), &mg, &s.p);
            if (st != TPO_OK) return fail_with(s, st);
            std::memcpy(s.dims, dims, sizeof(dims));
            s.Ke64 = Ke;
            s.fixed = fixed;
        }
        st = tpo_set_densities(s.p, q.densities, q.penal, q.E0, q.Emin);
        if (st != TPO_OK) return fail_with(s, st);
        std::vector<double> F(q.F, q.F + q.ndof);
        st = tpo_set_load(s.p, F.data());
        if (st != TPO_OK) return fail_with(s, st);
    } else {
        seam_destroy(s);
        s.Ke64 = Ke;
        s.dens64.assign(q.densities, q.densities + q.nel);
        s.F64.assign(q.F, q.F + q.ndof);
        s.edofs.assign(q.edofArray, q.edofArray + q.nel * 24);
        s.freedofs.clear();
        for (int64_t i = 0; i < q.ndof; i++)
            if (!q.fixedMask[i]) s.freedofs.push_back((int32_t)i);
    }
    s.structured = structured;
    s.ready = true;
    return TPO_OK;
}

// GPUFEASolver.solve: U (ndof floats) written, as the reference returns a Float32Array;
// U64 (optional) receives the FP64 solution.  TPO_NOT_CONVERGED is not an error: the
// reference reports converged = false with the iterate.
inline tpo_status seam_solve(State &s, int maxIterations, double tolerance, const float *warmStart, float *U,
                             double *U64, int *iterations, int *converged) {
    if (!s.ready) {
        s.error = "GPUFEASolver: not initialized. Call init() and setup() first.";
        return TPO_BAD_ARG;
    }
    std::vector<double> u((size_t)s.ndof, 0.0);
    if (warmStart)
        for (int64_t i = 0; i < s.ndof; i++) u[i] = warmStart[i];
    tpo_status st;
    int its = 0, conv = 0;
    if (s.structured) {
        tpo_solve_opts o;
        tpo_default_solve_opts(&o);
        o.precond = s.solver_mg ? TPO_PREC_MG : TPO_PREC_JACOBI;
        o.precision = TPO_FP64;
        o.max_iter = maxIterations;
        o.tol = tolerance;
        o.warm_start = 1;
        o.ref_epsilon = 1;
        tpo_solve_info info{};
        st = tpo_solve(s.p, &o, u.data(), &info);
        its = info.iterations;
        conv = info.converged;
    } else {
        int32_t it = 0;
        st = tpo_ebe_pcg(s.dens64.data(), s.Ke64.data(), s.edofs.data(), s.F64.data(), u.data(), s.freedofs.data(),
                         (int32_t)s.nel, 24, (int32_t)s.ndof, (int32_t)s.freedofs.size(), s.Emin, s.E0, s.penal,
                         maxIterations, tolerance, &it);
        its = it;
        conv = st == TPO_OK;
    }
    if (st != TPO_OK && st != TPO_NOT_CONVERGED) return fail_with(s, st);
    for (int64_t i = 0; i < s.ndof; i++) U[i] = (float)u[i];
    if (U64) std::memcpy(U64, u.data(), (size_t)s.ndof * sizeof(double));
    if (iterations) *iterations = its;
    if (converged) *converged = conv;
    return TPO_OK;
}

// One SIMP iteration on the device problem of the last setup (tpo_simp_step): the body of
// the worker's loop (js/optimizer-worker-3d.js:2074-2301: projection, FE solve, energies,
// sensitivities, filter, OC, change) in one call, so a JavaScript loop that keeps only its
// control (penal continuation, beta and tolerance schedules) makes one call per iteration.
// x (nel floats) is updated in place; preserved / voidm (nel bytes) may be null.  The
// solver is the setup's (the reference's Jacobi-PCG, or MG-PCG with solver 'mgpcg'),
// cold-started for MG-PCG and warm-started for Jacobi-PCG as the worker does.
struct SimpParams {
    double volfrac = 0.3, penal = 3.0, rmin = 1.5, beta = 1.0, tolerance = 1e-8;
    int use_projection = 0, max_iterations = 400, warm_start = 1;
};
inline tpo_status seam_simp_step(State &s, const SimpParams &q, float *x, const uint8_t *preserved,
                                 const uint8_t *voidm, double *compliance, double *change, int *cg_iterations) {
    if (!s.ready || !s.structured || !s.p) {
        s.error = "simpStep: needs setup() on the worker's structured numbering first";
        return TPO_BAD_ARG;
    }
    tpo_simp_opts o;
    std::memset(&o, 0, sizeof o);
    o.volfrac = q.volfrac;
    o.penal = q.penal;
    o.rmin = q.rmin;
    o.E0 = s.E0;
    o.Emin = s.Emin;
    o.beta = q.beta;
    o.use_projection = q.use_projection;
    o.guard_sensitivities = 0;
    tpo_default_solve_opts(&o.solve);
    o.solve.precond = s.solver_mg ? TPO_PREC_MG : TPO_PREC_JACOBI;
    o.solve.precision = TPO_FP64;
    o.solve.max_iter = q.max_iterations;
    o.solve.tol = q.tolerance;
    o.solve.warm_start = s.solver_mg ? 0 : q.warm_start;
    o.solve.ref_epsilon = 1;
    tpo_simp_info info{};
    const tpo_status st = tpo_simp_step(s.p, &o, x, preserved, voidm, &info);
    if (st != TPO_OK) return fail_with(s, st);
    if (compliance) *compliance = info.compliance;
    if (change) *change = info.change;
    if (cg_iterations) *cg_iterations = info.cg_iterations;
    return TPO_OK;
}

// ebeKSP_BDDC (assembly/index.ts:1385-1404) as _solveWithWasmKSP_BDDC calls it
// (js/optimizer-worker-3d.js:3814-3970): a structured nelx x nely x nelz grid with its
// densities, supports and load, cold start, the worker's smoother count
// (KSP_BDDC_SMOOTHER_ITERS = 3, :1031).  The subdomains the worker builds
// (KSPSolver._buildSubdomains, :1141-1231) are built on the device from the grid.  The
// preconditioner is indefinite for this element matrix, so the solve reports
// TPO_NOT_CONVERGED after maxIter iterations as a rule; that is not an error, as the WASM
// call returns its iteration count either way.
inline tpo_status seam_ksp_bddc(const int dims[3], const double *Ke, const float *densities, double penal, double E0,
                                double Emin, const uint8_t *fixedMask, const double *F, double *U, int maxIter,
                                double tol, int smootherIters, int *iterations, std::string *error) {
    tpo_mg_opts mg;
    tpo_default_mg_opts(&mg);
    const tpo_grid g{dims[0], dims[1], dims[2]};
    tpo_problem *p = nullptr;
    tpo_status st = tpo_create(&g, Ke, 0.3, fixedMask, &mg, &p);
    if (st == TPO_OK) st = tpo_set_densities(p, densities, penal, E0, Emin);
    int32_t it = 0;
    if (st == TPO_OK) st = tpo_ksp_bddc(p, F, U, maxIter, tol, smootherIters, &it);
    if (iterations) *iterations = it;
    if (st != TPO_OK && st != TPO_NOT_CONVERGED && error) {
        const char *m = tpo_last_error();
        *error = std::string(tpo_status_string(st)) + ": " + (m ? m : "");
    }
    if (p) tpo_destroy(p);
    return st == TPO_NOT_CONVERGED ? TPO_OK : st;
}

}  // namespace tpo_seam
