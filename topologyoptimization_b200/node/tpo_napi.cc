// tpo_napi.cc -- Node-API binding of libtpo for the reference's JavaScript worker.
//
// Not built in this repository's environment (it has no Node runtime or node_api.h); a
// maintainer builds it with node-gyp (binding.gyp beside this file).  The call sequence of
// setup / solve lives in tpo_seam.h, which tests/harness/seam_harness.cc drives on a GPU.
//
// Exports (each mirrors one seam of js/optimizer-worker-3d.js):
//   deviceAvailable() -> bool                            GPUFEASolver.init (js/gpu-fea-solver.js:91-141)
//   setup(handle | null, params) -> handle               GPUFEASolver.setup (:162-191)
//   solve(handle, maxIterations, tolerance, warmStart | null)
//        -> Promise<{U: Float32Array, iterations, converged}>   GPUFEASolver.solve (:704-820)
//   destroy(handle)                                       GPUFEASolver.destroy (:836-845)
//   ebePCG(dens, KEflat, edofs, F, U, freedofs, nel, edofSize, ndof, nfree, Emin, E0, penal,
//          maxIter, tol) -> iterations                    assembly/index.ts:504-733
//   applyAEbe3D(KEflat, edofs, evals, active, activeCount, p, Ap, ndof)   :403-439
//   denseMatVecRaw(K, p, Ap, n)                           :450-464
//   ebeKSP_BDDC(nelx, nely, nelz, KEflat, densities, penal, E0, Emin, fixedMask, F, U,
//               maxIter, tol, smootherIters) -> iterations     :1385-1404
//   simpStep(handle, options, x, preserved | null, void | null)
//        -> {compliance, change, cgIterations}             one iteration of the worker's loop
//   computeElementEnergies(U, KEflat, edofs, nel, edofSize) -> Float32Array
//                                                         GPUCompute (js/gpu-compute.js:187-303)
//   forward(handle, design, x, l | null) -> Promise<number>          chosen form: objective
//   backward(handle, l | null) -> Promise<Float64Array>              chosen form: dJ/dx
//
// Typed arrays are passed to libtpo as raw pointers (no copy on the JavaScript side).  A
// failing status throws an Error with tpo_last_error(); the worker catches it and falls
// back to WASM/JS (js/optimizer-worker-3d.js:4149-4152).  TPO_NOT_CONVERGED is not an
// error: the result reports converged = false.
#include <node_api.h>

#include <cstring>
#include <string>
#include <vector>

#include "tpo.h"
#include "tpo_seam.h"

namespace {

#define NAPI_OK(call)                                                   \
    do {                                                                \
        if ((call) != napi_ok) {                                        \
            napi_throw_error(env, nullptr, "tpo_napi: N-API call failed"); \
            return nullptr;                                             \
        }                                                               \
    } while (0)

napi_value throw_status(napi_env env, tpo_status st, const std::string &where) {
    const std::string msg = where + ": " + tpo_status_string(st) + ": " + tpo_last_error();
    napi_throw_error(env, nullptr, msg.c_str());
    return nullptr;
}

// Pointer and element count of a typed array argument (nullptr for null / undefined).
bool typed(napi_env env, napi_value v, void **data, size_t *len, napi_typedarray_type want) {
    napi_valuetype vt;
    if (napi_typeof(env, v, &vt) != napi_ok) return false;
    if (vt == napi_null || vt == napi_undefined) {
        *data = nullptr;
        *len = 0;
        return true;
    }
    bool is_ta = false;
    if (napi_is_typedarray(env, v, &is_ta) != napi_ok || !is_ta) return false;
    napi_typedarray_type t;
    napi_value ab;
    size_t off;
    if (napi_get_typedarray_info(env, v, &t, len, data, &ab, &off) != napi_ok) return false;
    return t == want;
}

bool prop_typed(napi_env env, napi_value obj, const char *key, void **data, size_t *len, napi_typedarray_type want) {
    napi_value v;
    if (napi_get_named_property(env, obj, key, &v) != napi_ok) return false;
    return typed(env, v, data, len, want);
}

double prop_number(napi_env env, napi_value obj, const char *key, double dflt) {
    bool has = false;
    if (napi_has_named_property(env, obj, key, &has) != napi_ok || !has) return dflt;
    napi_value v;
    double d = dflt;
    if (napi_get_named_property(env, obj, key, &v) == napi_ok) napi_get_value_double(env, v, &d);
    return d;
}

std::string prop_string(napi_env env, napi_value obj, const char *key) {
    bool has = false;
    if (napi_has_named_property(env, obj, key, &has) != napi_ok || !has) return "";
    napi_value v;
    char buf[64] = {0};
    size_t n = 0;
    if (napi_get_named_property(env, obj, key, &v) != napi_ok) return "";
    if (napi_get_value_string_utf8(env, v, buf, sizeof(buf), &n) != napi_ok) return "";
    return std::string(buf, n);
}

double arg_number(napi_env env, napi_value v) {
    double d = 0.0;
    napi_get_value_double(env, v, &d);
    return d;
}

// ---- the solver handle -----------------------------------------------------------------
struct Handle {
    tpo_seam::State s;
};

void finalize_handle(napi_env, void *data, void *) {
    Handle *h = static_cast<Handle *>(data);
    tpo_seam::seam_destroy(h->s);
    delete h;
}

Handle *get_handle(napi_env env, napi_value v) {
    void *p = nullptr;
    napi_valuetype vt;
    if (napi_typeof(env, v, &vt) != napi_ok || vt != napi_external) return nullptr;
    if (napi_get_value_external(env, v, &p) != napi_ok) return nullptr;
    return static_cast<Handle *>(p);
}

napi_value DeviceAvailable(napi_env env, napi_callback_info) {
    napi_value v;
    NAPI_OK(napi_get_boolean(env, tpo_device_available() == 1, &v));
    return v;
}

// setup(handle | null, params): returns the handle (a new one when null).
napi_value Setup(napi_env env, napi_callback_info info) {
    size_t argc = 2;
    napi_value a[2];
    NAPI_OK(napi_get_cb_info(env, info, &argc, a, nullptr, nullptr));
    if (argc < 2) {
        napi_throw_error(env, nullptr, "setup(handle, params)");
        return nullptr;
    }
    napi_value hv = a[0];
    Handle *h = get_handle(env, a[0]);
    if (!h) {
        h = new Handle();
        NAPI_OK(napi_create_external(env, h, finalize_handle, nullptr, &hv));
    }
    tpo_seam::SetupParams q;
    size_t n = 0;
    void *d = nullptr;
    if (!prop_typed(env, a[1], "KEflat", &d, &n, napi_float32_array) || n != 576) {
        napi_throw_type_error(env, nullptr, "GPUFEASolver.setup: KEflat must be a Float32Array(576)");
        return nullptr;
    }
    q.KEflat = static_cast<const float *>(d);
    if (!prop_typed(env, a[1], "edofArray", &d, &n, napi_int32_array)) {
        napi_throw_type_error(env, nullptr, "GPUFEASolver.setup: edofArray must be an Int32Array");
        return nullptr;
    }
    q.edofArray = static_cast<const int32_t *>(d);
    const size_t n_edofs = n;
    if (!prop_typed(env, a[1], "densities", &d, &n, napi_float32_array)) {
        napi_throw_type_error(env, nullptr, "GPUFEASolver.setup: densities must be a Float32Array");
        return nullptr;
    }
    q.densities = static_cast<const float *>(d);
    const size_t n_dens = n;
    if (!prop_typed(env, a[1], "F", &d, &n, napi_float32_array)) {
        napi_throw_type_error(env, nullptr, "GPUFEASolver.setup: F must be a Float32Array");
        return nullptr;
    }
    q.F = static_cast<const float *>(d);
    const size_t n_F = n;
    if (!prop_typed(env, a[1], "fixedMask", &d, &n, napi_uint8_array)) {
        napi_throw_type_error(env, nullptr, "GPUFEASolver.setup: fixedMask must be a Uint8Array");
        return nullptr;
    }
    q.fixedMask = static_cast<const uint8_t *>(d);
    const size_t n_fix = n;
    q.nel = (int64_t)prop_number(env, a[1], "nel", 0);
    q.ndof = (int64_t)prop_number(env, a[1], "ndof", 0);
    q.E0 = prop_number(env, a[1], "E0", 1.0);
    q.Emin = prop_number(env, a[1], "Emin", 1e-9);
    q.penal = prop_number(env, a[1], "penal", 3.0);
    q.solver_mg = prop_string(env, a[1], "solver") == "mgpcg" ? 1 : 0;
    if (n_edofs != (size_t)q.nel * 24 || n_dens != (size_t)q.nel || n_F != (size_t)q.ndof ||
        n_fix != (size_t)q.ndof) {
        napi_throw_range_error(env, nullptr, "GPUFEASolver.setup: array lengths do not match nel / ndof");
        return nullptr;
    }
    const tpo_status st = tpo_seam::seam_setup(h->s, q);
    if (st != TPO_OK) {
        napi_throw_error(env, nullptr, h->s.error.c_str());
        return nullptr;
    }
    return hv;
}

// solve runs on the libuv pool (napi_async_work); the Promise resolves on the JS thread.
struct SolveWork {
    napi_async_work work = nullptr;
    napi_deferred deferred = nullptr;
    Handle *h = nullptr;
    napi_ref handle_ref = nullptr;  // keeps the handle alive while the work runs
    int max_it = 400;
    double tol = 1e-8;
    std::vector<float> warm;
    bool has_warm = false;
    std::vector<float> U;
    int iterations = 0, converged = 0;
    tpo_status st = TPO_OK;
    std::string error;
};

void solve_execute(napi_env, void *data) {
    SolveWork *w = static_cast<SolveWork *>(data);
    w->U.assign((size_t)w->h->s.ndof, 0.0f);
    w->st = tpo_seam::seam_solve(w->h->s, w->max_it, w->tol, w->has_warm ? w->warm.data() : nullptr, w->U.data(),
                                 nullptr, &w->iterations, &w->converged);
    if (w->st != TPO_OK) w->error = w->h->s.error;
}

void solve_complete(napi_env env, napi_status, void *data) {
    SolveWork *w = static_cast<SolveWork *>(data);
    if (w->st != TPO_OK) {
        napi_value msg, err;
        napi_create_string_utf8(env, w->error.c_str(), NAPI_AUTO_LENGTH, &msg);
        napi_create_error(env, nullptr, msg, &err);
        napi_reject_deferred(env, w->deferred, err);
    } else {
        napi_value res, ab, U, it, conv;
        void *buf = nullptr;
        const size_t n = w->U.size();
        napi_create_arraybuffer(env, n * sizeof(float), &buf, &ab);
        std::memcpy(buf, w->U.data(), n * sizeof(float));
        napi_create_typedarray(env, napi_float32_array, n, ab, 0, &U);
        napi_create_int32(env, w->iterations, &it);
        napi_get_boolean(env, w->converged != 0, &conv);
        napi_create_object(env, &res);
        napi_set_named_property(env, res, "U", U);
        napi_set_named_property(env, res, "iterations", it);
        napi_set_named_property(env, res, "converged", conv);
        napi_resolve_deferred(env, w->deferred, res);
    }
    napi_delete_reference(env, w->handle_ref);
    napi_delete_async_work(env, w->work);
    delete w;
}

// solve(handle, maxIterations, tolerance, warmStart | null) -> Promise
napi_value Solve(napi_env env, napi_callback_info info) {
    size_t argc = 4;
    napi_value a[4];
    NAPI_OK(napi_get_cb_info(env, info, &argc, a, nullptr, nullptr));
    Handle *h = argc >= 1 ? get_handle(env, a[0]) : nullptr;
    if (!h || !h->s.ready) {
        napi_throw_error(env, nullptr, "GPUFEASolver: not initialized. Call init() and setup() first.");
        return nullptr;
    }
    SolveWork *w = new SolveWork();
    w->h = h;
    w->max_it = argc >= 2 ? (int)arg_number(env, a[1]) : 400;
    w->tol = argc >= 3 ? arg_number(env, a[2]) : 1e-8;
    if (argc >= 4) {
        void *d = nullptr;
        size_t n = 0;
        if (!typed(env, a[3], &d, &n, napi_float32_array) || (d && n != (size_t)h->s.ndof)) {
            delete w;
            napi_throw_type_error(env, nullptr, "GPUFEASolver.solve: warmStart must be a Float32Array(ndof)");
            return nullptr;
        }
        if (d) {
            w->warm.assign(static_cast<const float *>(d), static_cast<const float *>(d) + n);
            w->has_warm = true;
        }
    }
    napi_value promise, name;
    NAPI_OK(napi_create_promise(env, &w->deferred, &promise));
    NAPI_OK(napi_create_reference(env, a[0], 1, &w->handle_ref));
    NAPI_OK(napi_create_string_utf8(env, "tpo_solve", NAPI_AUTO_LENGTH, &name));
    NAPI_OK(napi_create_async_work(env, nullptr, name, solve_execute, solve_complete, w, &w->work));
    NAPI_OK(napi_queue_async_work(env, w->work));
    return promise;
}

napi_value Destroy(napi_env env, napi_callback_info info) {
    size_t argc = 1;
    napi_value a[1];
    NAPI_OK(napi_get_cb_info(env, info, &argc, a, nullptr, nullptr));
    Handle *h = argc >= 1 ? get_handle(env, a[0]) : nullptr;
    if (h) tpo_seam::seam_destroy(h->s);  // the external's finaliser frees the struct
    napi_value u;
    NAPI_OK(napi_get_undefined(env, &u));
    return u;
}

// ---- the WASM export surface (synchronous, as the WASM calls are) ------------------------
napi_value EbePCG(napi_env env, napi_callback_info info) {
    size_t argc = 15;
    napi_value a[15];
    NAPI_OK(napi_get_cb_info(env, info, &argc, a, nullptr, nullptr));
    if (argc < 15) {
        napi_throw_error(env, nullptr, "ebePCG: 15 arguments expected");
        return nullptr;
    }
    void *dens, *ke, *ed, *F, *U, *fr;
    size_t ndens, nke, ned, nF, nU, nfr;
    if (!typed(env, a[0], &dens, &ndens, napi_float64_array) || !typed(env, a[1], &ke, &nke, napi_float64_array) ||
        !typed(env, a[2], &ed, &ned, napi_int32_array) || !typed(env, a[3], &F, &nF, napi_float64_array) ||
        !typed(env, a[4], &U, &nU, napi_float64_array) || !typed(env, a[5], &fr, &nfr, napi_int32_array)) {
        napi_throw_type_error(env, nullptr, "ebePCG: typed array arguments expected");
        return nullptr;
    }
    const int32_t nel = (int32_t)arg_number(env, a[6]), es = (int32_t)arg_number(env, a[7]);
    const int32_t ndof = (int32_t)arg_number(env, a[8]), nfree = (int32_t)arg_number(env, a[9]);
    if (ndens < (size_t)nel || nke < (size_t)es * es || ned < (size_t)nel * es || nF < (size_t)ndof ||
        nU < (size_t)ndof || nfr < (size_t)nfree) {
        napi_throw_range_error(env, nullptr, "ebePCG: an array is shorter than its size argument");
        return nullptr;
    }
    int32_t it = 0;
    const tpo_status st = tpo_ebe_pcg(static_cast<double *>(dens), static_cast<double *>(ke), static_cast<int32_t *>(ed),
                                      static_cast<double *>(F), static_cast<double *>(U), static_cast<int32_t *>(fr), nel,
                                      es, ndof, nfree, arg_number(env, a[10]), arg_number(env, a[11]),
                                      arg_number(env, a[12]), (int32_t)arg_number(env, a[13]), arg_number(env, a[14]),
                                      &it);
    if (st != TPO_OK && st != TPO_NOT_CONVERGED) return throw_status(env, st, "ebePCG");
    napi_value r;
    NAPI_OK(napi_create_int32(env, it, &r));
    return r;
}

// simpStep(handle, {volfrac, penal, rmin, beta, useProjection, tolerance, maxIterations},
//          x: Float32Array(nel), preserved: Uint8Array | null, void: Uint8Array | null)
//   -> {compliance, change, cgIterations}; x is updated in place.
napi_value SimpStep(napi_env env, napi_callback_info info) {
    size_t argc = 5;
    napi_value a[5];
    NAPI_OK(napi_get_cb_info(env, info, &argc, a, nullptr, nullptr));
    Handle *h = argc >= 5 ? get_handle(env, a[0]) : nullptr;
    if (!h) {
        napi_throw_type_error(env, nullptr, "simpStep: (handle, options, x, preserved, void) expected");
        return nullptr;
    }
    void *x, *pres, *vd;
    size_t nx, np_, nv;
    if (!typed(env, a[2], &x, &nx, napi_float32_array) || !x || !typed(env, a[3], &pres, &np_, napi_uint8_array) ||
        !typed(env, a[4], &vd, &nv, napi_uint8_array)) {
        napi_throw_type_error(env, nullptr, "simpStep: x must be a Float32Array, the masks Uint8Array or null");
        return nullptr;
    }
    const size_t nel = (size_t)h->s.nel;
    if (nx != nel || (pres && np_ != nel) || (vd && nv != nel)) {
        napi_throw_range_error(env, nullptr, "simpStep: arrays must have nel entries");
        return nullptr;
    }
    tpo_seam::SimpParams q;
    q.volfrac = prop_number(env, a[1], "volfrac", q.volfrac);
    q.penal = prop_number(env, a[1], "penal", q.penal);
    q.rmin = prop_number(env, a[1], "rmin", q.rmin);
    q.beta = prop_number(env, a[1], "beta", q.beta);
    q.use_projection = (int)prop_number(env, a[1], "useProjection", 0);
    q.tolerance = prop_number(env, a[1], "tolerance", q.tolerance);
    q.max_iterations = (int)prop_number(env, a[1], "maxIterations", q.max_iterations);
    double c = 0.0, ch = 0.0;
    int cg = 0;
    const tpo_status st = tpo_seam::seam_simp_step(h->s, q, static_cast<float *>(x), static_cast<uint8_t *>(pres),
                                                   static_cast<uint8_t *>(vd), &c, &ch, &cg);
    if (st != TPO_OK) {
        napi_throw_error(env, nullptr, h->s.error.c_str());
        return nullptr;
    }
    napi_value r, v;
    NAPI_OK(napi_create_object(env, &r));
    NAPI_OK(napi_create_double(env, c, &v));
    NAPI_OK(napi_set_named_property(env, r, "compliance", v));
    NAPI_OK(napi_create_double(env, ch, &v));
    NAPI_OK(napi_set_named_property(env, r, "change", v));
    NAPI_OK(napi_create_int32(env, cg, &v));
    NAPI_OK(napi_set_named_property(env, r, "cgIterations", v));
    return r;
}

napi_value KspBDDC(napi_env env, napi_callback_info info) {
    size_t argc = 14;
    napi_value a[14];
    NAPI_OK(napi_get_cb_info(env, info, &argc, a, nullptr, nullptr));
    if (argc < 14) {
        napi_throw_error(env, nullptr, "ebeKSP_BDDC: 14 arguments expected");
        return nullptr;
    }
    const int dims[3] = {(int)arg_number(env, a[0]), (int)arg_number(env, a[1]), (int)arg_number(env, a[2])};
    void *ke, *dens, *fix, *F, *U;
    size_t nke, ndens, nfix, nF, nU;
    if (!typed(env, a[3], &ke, &nke, napi_float64_array) || !typed(env, a[4], &dens, &ndens, napi_float32_array) ||
        !typed(env, a[8], &fix, &nfix, napi_uint8_array) || !typed(env, a[9], &F, &nF, napi_float64_array) ||
        !typed(env, a[10], &U, &nU, napi_float64_array)) {
        napi_throw_type_error(env, nullptr, "ebeKSP_BDDC: typed array arguments expected");
        return nullptr;
    }
    if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1) {
        napi_throw_range_error(env, nullptr, "ebeKSP_BDDC: grid sizes must be positive");
        return nullptr;
    }
    const size_t nel = (size_t)dims[0] * dims[1] * dims[2];
    const size_t ndof = 3 * (size_t)(dims[0] + 1) * (dims[1] + 1) * (dims[2] + 1);
    if (nke < 576 || ndens < nel || nfix < ndof || nF < ndof || nU < ndof) {
        napi_throw_range_error(env, nullptr, "ebeKSP_BDDC: an array is shorter than the grid needs");
        return nullptr;
    }
    int it = 0;
    std::string err;
    const tpo_status st = tpo_seam::seam_ksp_bddc(
        dims, static_cast<double *>(ke), static_cast<float *>(dens), arg_number(env, a[5]), arg_number(env, a[6]),
        arg_number(env, a[7]), static_cast<uint8_t *>(fix), static_cast<double *>(F), static_cast<double *>(U),
        (int)arg_number(env, a[11]), arg_number(env, a[12]), (int)arg_number(env, a[13]), &it, &err);
    if (st != TPO_OK) {
        napi_throw_error(env, nullptr, err.c_str());
        return nullptr;
    }
    napi_value r;
    NAPI_OK(napi_create_int32(env, it, &r));
    return r;
}

napi_value ApplyAEbe3D(napi_env env, napi_callback_info info) {
    size_t argc = 8;
    napi_value a[8];
    NAPI_OK(napi_get_cb_info(env, info, &argc, a, nullptr, nullptr));
    void *ke, *ed, *ev, *act, *p, *ap;
    size_t nke, ned, nev, nact, np, nap;
    if (argc < 8 || !typed(env, a[0], &ke, &nke, napi_float64_array) || !typed(env, a[1], &ed, &ned, napi_int32_array) ||
        !typed(env, a[2], &ev, &nev, napi_float64_array) || !typed(env, a[3], &act, &nact, napi_int32_array) ||
        !typed(env, a[5], &p, &np, napi_float64_array) || !typed(env, a[6], &ap, &nap, napi_float64_array)) {
        napi_throw_type_error(env, nullptr, "applyAEbe3D(KEflat, edofs, evals, active, activeCount, p, Ap, ndof)");
        return nullptr;
    }
    const int32_t count = (int32_t)arg_number(env, a[4]), ndof = (int32_t)arg_number(env, a[7]);
    if (nke < 576 || nact < (size_t)count || np < (size_t)ndof || nap < (size_t)ndof || ned < nev * 24) {
        napi_throw_range_error(env, nullptr, "applyAEbe3D: an array is shorter than its size argument");
        return nullptr;
    }
    const tpo_status st =
        tpo_apply_a_ebe3d(static_cast<double *>(ke), static_cast<int32_t *>(ed), static_cast<double *>(ev),
                          static_cast<int32_t *>(act), count, (int32_t)nev, static_cast<double *>(p),
                          static_cast<double *>(ap), ndof);
    if (st != TPO_OK) return throw_status(env, st, "applyAEbe3D");
    napi_value u;
    NAPI_OK(napi_get_undefined(env, &u));
    return u;
}

napi_value DenseMatVecRaw(napi_env env, napi_callback_info info) {
    size_t argc = 4;
    napi_value a[4];
    NAPI_OK(napi_get_cb_info(env, info, &argc, a, nullptr, nullptr));
    void *K, *p, *ap;
    size_t nK, np, nap;
    if (argc < 4 || !typed(env, a[0], &K, &nK, napi_float64_array) || !typed(env, a[1], &p, &np, napi_float64_array) ||
        !typed(env, a[2], &ap, &nap, napi_float64_array)) {
        napi_throw_type_error(env, nullptr, "denseMatVecRaw(K, p, Ap, n)");
        return nullptr;
    }
    const int32_t n = (int32_t)arg_number(env, a[3]);
    if (nK < (size_t)n * n || np < (size_t)n || nap < (size_t)n) {
        napi_throw_range_error(env, nullptr, "denseMatVecRaw: an array is shorter than n");
        return nullptr;
    }
    const tpo_status st =
        tpo_dense_matvec(static_cast<double *>(K), static_cast<double *>(p), static_cast<double *>(ap), n);
    if (st != TPO_OK) return throw_status(env, st, "denseMatVecRaw");
    napi_value u;
    NAPI_OK(napi_get_undefined(env, &u));
    return u;
}

// computeElementEnergies(U, KEflat, edofs, nel, edofSize) -> Float32Array (synchronous
// here; the shim wraps it in a Promise as GPUCompute's method is async)
napi_value ComputeElementEnergies(napi_env env, napi_callback_info info) {
    size_t argc = 5;
    napi_value a[5];
    NAPI_OK(napi_get_cb_info(env, info, &argc, a, nullptr, nullptr));
    void *U, *ke, *ed;
    size_t nU, nke, ned;
    if (argc < 5 || !typed(env, a[0], &U, &nU, napi_float32_array) || !typed(env, a[1], &ke, &nke, napi_float32_array) ||
        !typed(env, a[2], &ed, &ned, napi_int32_array)) {
        napi_throw_type_error(env, nullptr, "computeElementEnergies(U, KEflat, edofs, nel, edofSize)");
        return nullptr;
    }
    const int32_t nel = (int32_t)arg_number(env, a[3]), es = (int32_t)arg_number(env, a[4]);
    if (ned < (size_t)nel * es || nke < (size_t)es * es) {
        napi_throw_range_error(env, nullptr, "computeElementEnergies: an array is shorter than its size arguments");
        return nullptr;
    }
    napi_value ab, out;
    void *buf = nullptr;
    NAPI_OK(napi_create_arraybuffer(env, (size_t)nel * sizeof(float), &buf, &ab));
    const tpo_status st = tpo_element_energies(static_cast<float *>(U), static_cast<float *>(ke),
                                               static_cast<int32_t *>(ed), nel, es, (int32_t)nU, static_cast<float *>(buf));
    if (st != TPO_OK) return throw_status(env, st, "computeElementEnergies");
    NAPI_OK(napi_create_typedarray(env, napi_float32_array, (size_t)nel, ab, 0, &out));
    return out;
}

// ---- forward / backward (the chosen form's differentiable objective) ----------------------
struct AdjWork {
    napi_async_work work = nullptr;
    napi_deferred deferred = nullptr;
    napi_ref handle_ref = nullptr;
    Handle *h = nullptr;
    bool backward = false;
    tpo_design_opts design{};
    std::vector<double> x, l, grad;
    bool has_l = false;
    double J = 0.0;
    tpo_status st = TPO_OK;
    std::string error;
};

tpo_solve_opts adjoint_solve_opts() {
    tpo_solve_opts o;
    tpo_default_solve_opts(&o);
    o.precond = TPO_PREC_MG;
    o.precision = TPO_FP64;
    o.max_iter = 4000;
    o.tol = 1e-10;
    o.warm_start = 0;
    o.ref_epsilon = 0;
    return o;
}

void adj_execute(napi_env, void *data) {
    AdjWork *w = static_cast<AdjWork *>(data);
    const tpo_solve_opts o = adjoint_solve_opts();
    tpo_solve_info inf{};
    if (!w->backward) {
        w->st = tpo_forward(w->h->s.p, &w->design, &o, w->x.data(), w->has_l ? w->l.data() : nullptr, &w->J, &inf);
    } else {
        w->grad.assign((size_t)w->h->s.nel, 0.0);
        w->st = tpo_backward(w->h->s.p, &o, w->has_l ? w->l.data() : nullptr, w->grad.data(), &inf);
    }
    if (w->st != TPO_OK) w->error = std::string(tpo_status_string(w->st)) + ": " + tpo_last_error();
}

void adj_complete(napi_env env, napi_status, void *data) {
    AdjWork *w = static_cast<AdjWork *>(data);
    if (w->st != TPO_OK) {
        napi_value msg, err;
        napi_create_string_utf8(env, w->error.c_str(), NAPI_AUTO_LENGTH, &msg);
        napi_create_error(env, nullptr, msg, &err);
        napi_reject_deferred(env, w->deferred, err);
    } else if (!w->backward) {
        napi_value J;
        napi_create_double(env, w->J, &J);
        napi_resolve_deferred(env, w->deferred, J);
    } else {
        napi_value ab, g;
        void *buf = nullptr;
        napi_create_arraybuffer(env, w->grad.size() * sizeof(double), &buf, &ab);
        std::memcpy(buf, w->grad.data(), w->grad.size() * sizeof(double));
        napi_create_typedarray(env, napi_float64_array, w->grad.size(), ab, 0, &g);
        napi_resolve_deferred(env, w->deferred, g);
    }
    napi_delete_reference(env, w->handle_ref);
    napi_delete_async_work(env, w->work);
    delete w;
}

napi_value queue_adj(napi_env env, napi_value handle, AdjWork *w) {
    napi_value promise, name;
    NAPI_OK(napi_create_promise(env, &w->deferred, &promise));
    NAPI_OK(napi_create_reference(env, handle, 1, &w->handle_ref));
    NAPI_OK(napi_create_string_utf8(env, "tpo_adjoint", NAPI_AUTO_LENGTH, &name));
    NAPI_OK(napi_create_async_work(env, nullptr, name, adj_execute, adj_complete, w, &w->work));
    NAPI_OK(napi_queue_async_work(env, w->work));
    return promise;
}

bool read_l(napi_env env, napi_value v, AdjWork *w) {
    void *d = nullptr;
    size_t n = 0;
    if (!typed(env, v, &d, &n, napi_float64_array)) return false;
    if (d) {
        if (n != (size_t)w->h->s.ndof) return false;
        w->l.assign(static_cast<double *>(d), static_cast<double *>(d) + n);
        w->has_l = true;
    }
    return true;
}

// forward(handle, {penal, E0, Emin, filterRadius}, x: Float64Array(nel), l | null) -> Promise<J>
napi_value Forward(napi_env env, napi_callback_info info) {
    size_t argc = 4;
    napi_value a[4];
    NAPI_OK(napi_get_cb_info(env, info, &argc, a, nullptr, nullptr));
    Handle *h = argc >= 3 ? get_handle(env, a[0]) : nullptr;
    if (!h || !h->s.ready || !h->s.structured) {
        napi_throw_error(env, nullptr, "forward: needs a handle set up on a structured grid");
        return nullptr;
    }
    AdjWork *w = new AdjWork();
    w->h = h;
    w->design.penal = prop_number(env, a[1], "penal", 3.0);
    w->design.E0 = prop_number(env, a[1], "E0", 1.0);
    w->design.Emin = prop_number(env, a[1], "Emin", 1e-9);
    w->design.filter_radius = prop_number(env, a[1], "filterRadius", 0.0);
    void *d = nullptr;
    size_t n = 0;
    if (!typed(env, a[2], &d, &n, napi_float64_array) || !d || n != (size_t)h->s.nel ||
        (argc >= 4 && !read_l(env, a[3], w))) {
        delete w;
        napi_throw_type_error(env, nullptr, "forward: x must be a Float64Array(nel), l a Float64Array(ndof) or null");
        return nullptr;
    }
    w->x.assign(static_cast<double *>(d), static_cast<double *>(d) + n);
    return queue_adj(env, a[0], w);
}

// backward(handle, l | null) -> Promise<Float64Array(nel)> = dJ/dx of the last forward
napi_value Backward(napi_env env, napi_callback_info info) {
    size_t argc = 2;
    napi_value a[2];
    NAPI_OK(napi_get_cb_info(env, info, &argc, a, nullptr, nullptr));
    Handle *h = argc >= 1 ? get_handle(env, a[0]) : nullptr;
    if (!h || !h->s.ready || !h->s.structured) {
        napi_throw_error(env, nullptr, "backward: needs a handle set up on a structured grid");
        return nullptr;
    }
    AdjWork *w = new AdjWork();
    w->h = h;
    w->backward = true;
    if (argc >= 2 && !read_l(env, a[1], w)) {
        delete w;
        napi_throw_type_error(env, nullptr, "backward: l must be a Float64Array(ndof) or null");
        return nullptr;
    }
    return queue_adj(env, a[0], w);
}

napi_value Init(napi_env env, napi_value exports) {
    const napi_property_descriptor props[] = {
        {"deviceAvailable", nullptr, DeviceAvailable, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"setup", nullptr, Setup, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"solve", nullptr, Solve, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"destroy", nullptr, Destroy, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"ebePCG", nullptr, EbePCG, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"applyAEbe3D", nullptr, ApplyAEbe3D, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"denseMatVecRaw", nullptr, DenseMatVecRaw, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"ebeKSP_BDDC", nullptr, KspBDDC, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"simpStep", nullptr, SimpStep, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"computeElementEnergies", nullptr, ComputeElementEnergies, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"forward", nullptr, Forward, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"backward", nullptr, Backward, nullptr, nullptr, nullptr, napi_default, nullptr},
    };
    if (napi_define_properties(env, exports, sizeof(props) / sizeof(props[0]), props) != napi_ok) return nullptr;
    return exports;
}

}  // namespace

NAPI_MODULE(NODE_GYP_MODULE_NAME, Init)
