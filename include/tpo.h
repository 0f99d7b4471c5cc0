/*
 * tpo.h -- C ABI of libtpo.so, the B200 (sm_100a) implementation of the 3D SIMP
 * finite-element path of Jozo132/TopologyOptimization.
 *
 * Conventions (identical to the reference):
 *   - structured grid of unit hex8 elements, nelx x nely x nelz;
 *   - element e = ex + ey*nelx + ez*nelx*nely (x fastest);
 *   - node n = x*(nely+1)*(nelz+1) + y*(nelz+1) + z (z fastest), DOF = 3n + {0,1,2};
 *   - Ke is the 24x24 row-major element matrix in the local node order of
 *     js/optimizer-worker-3d.js:3404-3491.
 *
 * Every entry point returns a tpo_status and never aborts.  Host arrays are borrowed
 * for the duration of the call.  Functions whose name ends in _dev take device
 * pointers and run on the problem's stream.  One problem handle is used by one host
 * thread at a time.
 */
#ifndef TPO_H
#define TPO_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    TPO_OK = 0,
    TPO_NOT_CONVERGED = 1, /* iteration cap reached; the result is still written */
    TPO_NONFINITE = 2,     /* a NaN/Inf was detected in a residual or dot product */
    TPO_OOM = 3,           /* device allocation failed */
    TPO_BAD_ARG = 4,       /* invalid size, null pointer or inconsistent input */
    TPO_CUDA_ERROR = 5,    /* a CUDA runtime call failed; see tpo_last_error() */
    TPO_NO_DEVICE = 6,     /* no usable sm_100 device */
    TPO_TIMEOUT = 7        /* a bounded device wait ran out */
} tpo_status;

/* ---- library / device ------------------------------------------------------ */
const char *tpo_status_string(tpo_status s);
/* Message of the last failing call on this thread ("" if none). */
const char *tpo_last_error(void);
/* 1 when an sm_100 device is present and usable.  Mirrors GPUFEASolver.init /
 * isAvailable (js/gpu-fea-solver.js:91-141). */
int tpo_device_available(void);
/* Number of kernels this library has launched in this process (graph replays count
 * every captured kernel).  Instrumentation for benchmarks. */
int64_t tpo_launch_count(void);
/* 24x24 hex8 element matrix for E = 1 and Poisson ratio nu, computed on the device.
 * Replaces lk() (js/optimizer-worker-3d.js:3404-3491). */
tpo_status tpo_lk(double nu, double *Ke576);

/* ---- WASM export surface (assembly/index.ts), host arrays ---------------------
 * Same argument meaning as the WASM exports, with typed host pointers in place of
 * byte offsets into linear memory.  Work happens on the device; no workspace
 * pointer is needed (the library owns its scratch). */

/* applyAEbe3D (assembly/index.ts:403-439): Ap = sum over active e of E_e*Ke*p_e.
 * nel is the length of evals (edofs holds nel*24 entries). */
tpo_status tpo_apply_a_ebe3d(const double *Ke, const int32_t *edofs, const double *evals,
                             const int32_t *active, int32_t activeCount, int32_t nel,
                             const double *p, double *Ap, int32_t ndof);
/* GPUCompute.computeElementEnergies (js/gpu-compute.js:187-303, called by the worker at
 * js/optimizer-worker-3d.js:2146-2152): energies[e] = sum_i sum_j U[d_i] KE[i][j] U[d_j]
 * over the element's DOF indices d (negative indices skipped), in float32 in that order,
 * as the reference's WGSL kernel computes it.  Host arrays: U (ndof floats), KE
 * (edofSize^2 floats), edofs (nel * edofSize), energies (nel floats, written). */
tpo_status tpo_element_energies(const float *U, const float *KE, const int32_t *edofs, int32_t nel,
                                int32_t edofSize, int32_t ndof, float *energies);
/* denseMatVecRaw (assembly/index.ts:450-464). */
tpo_status tpo_dense_matvec(const double *K, const double *p, double *Ap, int32_t n);
/* ebePCG (assembly/index.ts:504-733): Jacobi-PCG on the free DOFs, warm start from U.
 * *iters receives the reference's return value.  edofSize 24 (hex8) or 8 (quad4). */
tpo_status tpo_ebe_pcg(const double *dens, const double *Ke, const int32_t *edofs,
                       const double *F, double *U, const int32_t *freedofs, int32_t nel,
                       int32_t edofSize, int32_t ndof, int32_t nfree, double Emin, double E0,
                       double penal, int32_t maxIter, double tol, int32_t *iters);

/* ---- device-resident problem (GPUFEASolver seam, js/gpu-fea-solver.js:73-845) - */
typedef struct tpo_problem tpo_problem;

typedef struct {
    int32_t nelx, nely, nelz;
} tpo_grid;

/* TPO_PREC_BDDC: the reference's KSP "BDDC" preconditioner (ebeKSP_BDDC / bddcApply,
 * assembly/index.ts:1204-1517, with the subdomain partition of KSPSolver._buildSubdomains,
 * js/optimizer-worker-3d.js:1141-1187): averaged subdomain-local Jacobi, undamped global
 * Jacobi sweeps and a Jacobi correction on the subdomain-corner DOFs.  As in the
 * reference it is not symmetric positive definite for the hex8 element matrix (the
 * undamped sweeps amplify the upper spectrum of D^-1 K, lambda_max ~ 5.3), so CG with it
 * usually does not reduce the residual; it is provided for the worker's
 * linearSolver 'petsc' path. */
typedef enum { TPO_PREC_JACOBI = 0, TPO_PREC_MG = 1, TPO_PREC_BDDC = 2 } tpo_precond;
/* TPO_FP64: FP64 PCG.  TPO_MIXED: FP32 MG-PCG recurrence with FP64 dot products and FP64
 * reliable updates (defect correction).  TPO_F32_PRECOND: FP64 PCG whose multigrid
 * preconditioner (every V-cycle level) runs in FP32. */
typedef enum { TPO_FP64 = 0, TPO_MIXED = 1, TPO_F32_PRECOND = 2 } tpo_precision;

typedef struct {
    int32_t max_levels;        /* reference MG_MAX_LEVELS = 6 */
    int32_t galerkin_max_ndof; /* reference GALERKIN_MAX_NDOF = 3000 */
    int32_t nu1, nu2;          /* reference 2, 2 */
    double omega;              /* reference 0.5 */
    int32_t coarse_iters;      /* reference 30 (sweeps at the coarsest level) */
    int32_t coarse_direct;     /* 0 reference sweeps; 1 Cholesky at the coarsest level */
    int32_t safe_omega;        /* 0 reference (omega on every level); 1 per-level damping
                                  min(omega, 1.9 / bound on lambda_max(D^-1 A)), which keeps
                                  the V-cycle positive definite on high-contrast designs */
    int32_t chebyshev;         /* 0 reference (damped Jacobi); 1 Chebyshev polynomial smoothing
                                  on the structured levels (nu1 / nu2 sweeps, the same applies
                                  as Jacobi) over [kappa / cheb_ratio, kappa], kappa the bound
                                  on lambda_max(D^-1 A); dense levels keep damped Jacobi */
    double cheb_ratio;         /* kappa / lower end of the smoothed interval (default 16) */
} tpo_mg_opts;

typedef struct {
    tpo_precond precond;
    tpo_precision precision;
    int32_t max_iter;
    double tol;          /* relative: ||r||^2 < tol^2 * max(||r0||^2, 1e-30) */
    int32_t warm_start;  /* 1: start from U (ebePCG / FE semantics); 0: U = 0 (ebeMGPCG) */
    int32_t ref_epsilon; /* 1: alpha = rz/(pAp+1e-12), beta = rz'/(rz+1e-12) as the
                            reference; 0: no absolute shift (breakdown-guarded) */
    /* mixed precision only */
    double inner_tol;     /* drop of the FP32 residual between two FP64 reliable updates (0.1) */
    int32_t tensor_cores; /* tcgen05 element contractions on the fine level: 1 TF32 in the V-cycle
                             (smoother, residual), 2 also for the FP32 CG operator (TPO_MIXED;
                             TF32's 10-bit mantissa there slows or stalls convergence on
                             high-contrast fields), 3 and 4 the same with 3xTF32 (high/low
                             operand split, FP32-class accuracy), 5 BF16 in the V-cycle
                             (TPO_F32_PRECOND only) */
    int32_t bddc_smoother_iters; /* TPO_PREC_BDDC: applies per preconditioner application (the
                                    worker's KSP_BDDC_SMOOTHER_ITERS = 3) */
} tpo_solve_opts;

typedef struct {
    int32_t iterations;       /* reference-convention iteration count (FP32 iterations for mixed) */
    int32_t outer_iterations; /* mixed precision: FP64 reliable updates (defect corrections) */
    int32_t converged;
    double rel_residual;      /* sqrt(||r||^2 / ||r0||^2) at exit (FP64 true residual for mixed) */
    double compliance;        /* F . U */
} tpo_solve_info;

/* Fill the option structs with their defaults (the reference's hierarchy and solver).
 * Callers start from these and then set the fields they need: fields are added at the
 * end of the structs as the library grows, and a struct filled field by field leaves
 * a newer field undefined (for tpo_mg_opts, a nonzero chebyshev with cheb_ratio <= 1
 * returns TPO_BAD_ARG, any other value silently selects Chebyshev smoothing). */
void tpo_default_mg_opts(tpo_mg_opts *o);
void tpo_default_solve_opts(tpo_solve_opts *o);

/* Create a problem on the current device.  Ke may be NULL (then lk(nu) is used).
 * fixedMask has 3*(nelx+1)*(nely+1)*(nelz+1) entries (1 = fixed DOF). */
tpo_status tpo_create(const tpo_grid *g, const double *Ke, double nu, const uint8_t *fixedMask,
                      const tpo_mg_opts *mg, tpo_problem **out);
tpo_status tpo_destroy(tpo_problem *p);
/* Sizes: nel and ndof of the fine grid; number of multigrid levels built. */
tpo_status tpo_sizes(const tpo_problem *p, int64_t *nel, int64_t *ndof, int32_t *levels);

/* Multigrid level li (0 = fine): dims[5] = nelx, nely, nelz, ndof, dense (1 when the level
 * is a dense Galerkin operator).  The hierarchy of MGPrecond3D.ensure
 * (js/optimizer-worker-3d.js:408-442). */
tpo_status tpo_level_info(const tpo_problem *p, int32_t level, int32_t *dims);
/* Copy a dense level's operator (ndof x ndof, row-major) to host memory K: the Galerkin
 * product of _assembleGalerkinFromElements / _assembleGalerkinFromMatrix
 * (js/optimizer-worker-3d.js:628-699), summed in the reference's order. */
tpo_status tpo_level_dense(tpo_problem *p, int32_t level, double *K);

/* Densities (reference element order) -> E_e = Emin + x^penal (E0 - Emin), active
 * where E_e > 1000 Emin, Jacobi diagonals and the multigrid hierarchy
 * (MGPrecond3D.updateFromFine, js/optimizer-worker-3d.js:558-582). */
tpo_status tpo_set_densities(tpo_problem *p, const float *x, double penal, double E0, double Emin);
tpo_status tpo_set_densities_dev(tpo_problem *p, const float *d_x, double penal, double E0,
                                 double Emin);
tpo_status tpo_set_load(tpo_problem *p, const double *F);
tpo_status tpo_set_load_dev(tpo_problem *p, const double *d_F);

/* Ku = K(x) u over active elements (no masking), host or device arrays. */
tpo_status tpo_apply(tpo_problem *p, const double *u, double *Ku);
tpo_status tpo_apply_dev(tpo_problem *p, const double *d_u, double *d_Ku);
/* Ku in FP32 (the mixed-precision inner operator), device arrays. */
tpo_status tpo_apply_f32_dev(tpo_problem *p, const float *d_u, float *d_Ku);
/* Ku with the element contraction Ke*u_e on the tensor cores (TF32 operands, FP32
 * accumulation), device arrays. */
tpo_status tpo_apply_tf32_dev(tpo_problem *p, const float *d_u, float *d_Ku);
/* The same with 3xTF32 (Ke and E_e u_e split into TF32 high and low parts,
 * D = Ah Bh + Ah Bl + Al Bh): FP32-class accuracy on the tensor cores. */
tpo_status tpo_apply_3xtf32_dev(tpo_problem *p, const float *d_u, float *d_Ku);
/* The same with BF16 operands (kind::f16 MMAs, FP32 accumulation): Ke and E_e u_e rounded
 * to an 8-bit mantissa, half the operand bytes of TF32 (relative error ~1e-3). */
tpo_status tpo_apply_bf16_dev(tpo_problem *p, const float *d_u, float *d_Ku);
/* z = V-cycle(b) from z = 0 (reference mgVcycle), host arrays. */
tpo_status tpo_vcycle(tpo_problem *p, const double *b, double *z);
/* Solve K U = F.  U is in/out (warm start when opts->warm_start). */
tpo_status tpo_solve(tpo_problem *p, const tpo_solve_opts *o, double *U, tpo_solve_info *info);
tpo_status tpo_solve_dev(tpo_problem *p, const tpo_solve_opts *o, double *d_U,
                         tpo_solve_info *info);

/* ---- SIMP pieces (device arrays, reference element order) -------------------- */
/* energy_e = u_e^T Ke u_e with unit Ke over every element, stored as float
 * (js/optimizer-worker-3d.js:2163-2173). */
tpo_status tpo_element_energy_dev(tpo_problem *p, const double *d_U, float *d_energy);
/* xPhys = Heaviside(x; beta, eta = 0.5) (:3500-3509). */
tpo_status tpo_heaviside_dev(tpo_problem *p, const float *d_x, double beta, float *d_xPhys);
/* dc_e = -penal xPhys^(penal-1) E0 energy_e * dxPhys/dx (:2175-2192). */
tpo_status tpo_sensitivity_dev(tpo_problem *p, const float *d_x, const float *d_xPhys,
                               const float *d_energy, double penal, double E0, double beta,
                               int32_t use_projection, float *d_dc);
/* Sensitivity filter (prepareFilter/filterSensitivities :3006-3064), float in/out. */
tpo_status tpo_filter_sens_dev(tpo_problem *p, double rmin, const float *d_x, const float *d_dc,
                               float *d_dcn);
/* Density filter of assembly/index.ts:224-273, double in/out. */
tpo_status tpo_density_filter_dev(tpo_problem *p, double radius, const double *d_x, double *d_out);
/* Transpose of that density filter (the adjoint of xPhys = H x / Hs, used by the
 * chosen form's backward pass): out_j = sum_i H_ij g_i / Hs_i, double in/out, out must
 * not alias g.  The reference has no transpose (its 3D loop filters sensitivities). */
tpo_status tpo_density_filter_transpose_dev(tpo_problem *p, double radius, const double *d_g, double *d_out);
/* OC bisection (:3066-3101).  preserved / void masks may be NULL. */
tpo_status tpo_oc_dev(tpo_problem *p, const float *d_x, double volfrac, const float *d_dc,
                      const uint8_t *d_preserved, const uint8_t *d_void, float *d_xnew,
                      double *lmid, int32_t *bisections);

/* OC with the arguments of the reference's update step (OC :3066-3101 with its move
 * limit, and the change test :2244-2247): x_new = clamp(x sqrt(-dc / lambda)) within
 * x +- move, lambda by bisection on [0, 1e9] until (l2 - l1) / (l2 + l1) <= 1e-3;
 * *change = max |x_new - x|.  The volume of each bisection step is summed exactly
 * (independent of the summation order) and rounded once.  More than max_bisections
 * steps (the reference's loop needs at most ~1100) returns TPO_TIMEOUT.  d_xnew must
 * not alias d_x. */
tpo_status tpo_oc_update_dev(tpo_problem *p, const float *d_x, const float *d_dc,
                             const uint8_t *d_preserved, const uint8_t *d_void, double volfrac,
                             double move, int32_t max_bisections, float *d_xnew, double *change,
                             double *lmid, int32_t *bisections);

/* ---- one SIMP iteration, device resident (optimize() loop body :2074-2247) ------ */
typedef struct {
    double volfrac, penal, rmin, E0, Emin;
    double beta;           /* Heaviside sharpness (used when use_projection) */
    int32_t use_projection;
    int32_t guard_sensitivities; /* 1: clamp element energies at 0 before the sensitivities.
                                    0 (reference): a rounding-negative energy gives dc > 0,
                                    sqrt(-dc/lambda) = NaN in OC and a NaN density */
    tpo_solve_opts solve;
} tpo_simp_opts;
typedef struct {
    double compliance, change;
    int32_t cg_iterations;
    int32_t converged;
    double rel_residual;
} tpo_simp_info;
/* d_x (design, reference order, float) is updated in place; U is kept on the device
 * between calls (warm start) and can be read with tpo_get_u. */
tpo_status tpo_simp_step_dev(tpo_problem *p, const tpo_simp_opts *o, float *d_x,
                             const uint8_t *d_preserved, const uint8_t *d_void,
                             tpo_simp_info *info);
/* The same step on host arrays: x (nel floats, the design) is copied to the device,
 * updated there and copied back before the call returns; preserved / void (nel bytes)
 * may be NULL.  The per-iteration call of the worker's loop (optimize,
 * js/optimizer-worker-3d.js:2074-2301) for a binding that holds the design in a
 * Float32Array. */
tpo_status tpo_simp_step(tpo_problem *p, const tpo_simp_opts *o, float *x, const uint8_t *preserved,
                         const uint8_t *voidm, tpo_simp_info *info);
tpo_status tpo_get_u(tpo_problem *p, double *U);
/* The volumetric snapshot of the last tpo_simp_step_dev (_buildVolumetricSnapshot,
 * js/optimizer-worker-3d.js:1579-1593, field of :2180-2184 and :2254-2255): stress[e] =
 * (Emin + xPhys_e^penal (E0 - Emin)) * energy_e as float (nel entries, host, reference
 * element order) and *max_stress, the largest stress of the step (0 when none is
 * positive).  TPO_BAD_ARG before the first SIMP step. */
tpo_status tpo_volumetric_snapshot(tpo_problem *p, float *stress, double *max_stress);
/* The CUDA stream the problem's work runs on (cudaStream_t as void*). */
void *tpo_stream(tpo_problem *p);
/* Run the problem's work on a caller-owned stream from now on (NULL: back to the
 * library's own stream).  The caller keeps the stream alive while the problem uses it.
 * The library's own stream is ordered with the legacy default stream; a caller's
 * non-blocking stream is not, so the caller orders its own work on it. */
tpo_status tpo_set_stream(tpo_problem *p, void *stream);

/* ---- batched solves (the chosen form's block MG-PCG; the reference solves load cases one
 * at a time) ------------------------------------------------------------------------- */
/* Solve K U_k = F_k for nrhs right-hand sides at once (1..64): d_F and d_U hold nrhs
 * device vectors of ndof each, one after the other; every kernel of the iteration runs
 * over all right-hand sides (grid z), each with its own PCG scalars and convergence
 * test, and the iterations of converged ones are skipped.  Precision TPO_FP64 or
 * TPO_F32_PRECOND, multigrid preconditioner; warm_start takes d_U as the initial guesses.
 * infos[k] (optional, nrhs entries) receives each solve's iterations, residual and F_k.U_k. */
tpo_status tpo_solve_multi_dev(tpo_problem *p, const tpo_solve_opts *o, int32_t nrhs, const double *d_F,
                               double *d_U, tpo_solve_info *infos);

/* ---- differentiable forward / backward (the chosen form's adjoint; the reference has
 * only the compliance sensitivity of js/optimizer-worker-3d.js:2175-2192) ------------- */
typedef struct {
    double penal, E0, Emin;
    double filter_radius; /* density filter xPhys = H x / Hs with the stencil of the WASM
                             applyDensityFilter (assembly/index.ts:224-273); <= 0: xPhys = x */
} tpo_design_opts;
/* Grounded spring K + k e_dof e_dof^T at one fine-level DOF (dof = -1 removes it); applies
 * to every later apply and solve of the problem. */
tpo_status tpo_set_spring(tpo_problem *p, int64_t dof, double k);
/* Forward pass from an FP64 design d_x (nel, reference element order, device):
 * xPhys = filter(x), E = Emin + xPhys^penal (E0 - Emin), hierarchy, solve K u = F (U stays
 * on the device).  *objective = l.u for the device vector d_l (ndof), or F.u (the
 * compliance) when d_l is NULL.  TPO_NOT_CONVERGED if the solve did not converge. */
tpo_status tpo_forward_dev(tpo_problem *p, const tpo_design_opts *d, const tpo_solve_opts *o,
                           const double *d_x, const double *d_l, double *objective, tpo_solve_info *info);
/* Backward pass of the last forward pass: dJ/dx (nel, reference order, device) for
 * J = l.u.  d_l NULL: compliance (self-adjoint, no second solve); otherwise the adjoint
 * K lambda = l is solved with options o.  dJ/dxPhys_e = -p xPhys^(p-1) (E0 - Emin)
 * lambda_e^T Ke u_e, then the filter transpose; d_grad_phys (optional) receives dJ/dxPhys. */
tpo_status tpo_backward_dev(tpo_problem *p, const tpo_solve_opts *o, const double *d_l, double *d_grad,
                            double *d_grad_phys, tpo_solve_info *info);

/* Host-array forms of tpo_forward_dev / tpo_backward_dev for bindings without device
 * memory of their own (x, grad: nel doubles; l: ndof doubles or NULL); the problem
 * stages them in device buffers it owns. */
tpo_status tpo_forward(tpo_problem *p, const tpo_design_opts *d, const tpo_solve_opts *o, const double *x,
                       const double *l, double *objective, tpo_solve_info *info);
tpo_status tpo_backward(tpo_problem *p, const tpo_solve_opts *o, const double *l, double *grad,
                        tpo_solve_info *info);

/* ebeMGPCG (assembly/index.ts:1076-1193) on a problem handle: U = MG-PCG solution of
 * K U = F (host arrays, ndof each) from a cold start with the reference's recurrence
 * (absolute 1e-12 shifts) and the problem's hierarchy; *iters receives the reference's
 * return value.  The hierarchy the worker serialises into 80-byte level descriptors
 * (js/optimizer-worker-3d.js:3750-3771) is built on the device by tpo_create /
 * tpo_set_densities instead. */
tpo_status tpo_mgpcg(tpo_problem *p, const double *F, double *U, int32_t maxIter, double tol,
                     int32_t *iters);

/* ebeKSP_BDDC (assembly/index.ts:1385-1404; caller _solveWithWasmKSP_BDDC,
 * js/optimizer-worker-3d.js:3814-3970): CG with the reference's BDDC preconditioner on the
 * handle's densities, cold start, the reference's 1e-12 shifts; *iters is the WASM return
 * value.  The subdomain and corner descriptors the worker writes into linear memory
 * (KSPSolver._buildSubdomains, :1141-1231) are built on the device from the grid;
 * smootherIters is the worker's KSP_BDDC_SMOOTHER_ITERS (1..64). */
tpo_status tpo_ksp_bddc(tpo_problem *p, const double *F, double *U, int32_t maxIter, double tol,
                        int32_t smootherIters, int32_t *iters);

/* ---- the 2D worker (js/optimizer-worker.js, TopologyOptimizerWorker) -----------------
 * Structured nelx x nely grid of bilinear quads with the 2D worker's numbering: element
 * e = ely + elx*nely (column-major), node n = (nely+1)*x + y, DOF = 2n + {0,1}. */
typedef struct tpo_problem2d tpo_problem2d;
typedef struct {
    double volfrac, penal, rmin, E0, Emin;
    double beta;            /* Heaviside sharpness (used when use_projection) */
    int32_t use_projection;
    double cg_tol;          /* absolute: ||r||^2 < cg_tol^2 (the worker's iterTolerance) */
    int32_t cg_max_iter;    /* the worker's MAX_CG_ITERATIONS = 2000; min(nfree, .) is applied */
} tpo_simp2d_opts;
typedef struct {
    double compliance, change;
    int32_t cg_iterations;
} tpo_simp2d_info;
/* 8x8 quad element matrix lk() (js/optimizer-worker.js:1732-1767). */
tpo_status tpo_lk2d(double nu, double *Ke64);
/* Ke may be NULL (lk2d(nu)); fixedMask has 2*(nelx+1)*(nely+1) entries. */
tpo_status tpo_create2d(int32_t nelx, int32_t nely, const double *Ke, double nu, const uint8_t *fixedMask,
                        tpo_problem2d **out);
tpo_status tpo_destroy2d(tpo_problem2d *p);
tpo_status tpo_set_load2d(tpo_problem2d *p, const double *F);
/* One iteration of the 2D loop body (:600-700) on the device: Heaviside projection,
 * E by Math.pow, Jacobi-PCG from U = 0 (solveCG :1799-1873), element energies, the
 * sensitivities, the 2D sensitivity filter (:1391-1443) and OC (:1445-1492) with the
 * change test.  d_x (float, 2D element order) is updated in place; preserved / void masks
 * may be NULL. */
tpo_status tpo_simp2d_step_dev(tpo_problem2d *p, const tpo_simp2d_opts *o, float *d_x,
                               const uint8_t *d_preserved, const uint8_t *d_void, tpo_simp2d_info *info);
tpo_status tpo_get_u2d(tpo_problem2d *p, double *U);

/* ---- allocation-free structured apply (no counterpart in the reference) ------------
 * Ku = K(x) u on a structured nelx*nely*nelz hex8 grid, for callers that must not
 * allocate device memory: no problem handle, no cudaMalloc/cudaFree, no library
 * allocator.  Same result as tpo_create + tpo_set_densities_dev(x, penal, E0, Emin) +
 * tpo_apply_dev(u, Ku) (E = Emin + x^penal (E0 - Emin), elements with E <= 1000 Emin
 * inactive; fixed DOFs are not masked).  Ke is a host 24x24 hex8 element matrix of
 * lk(nu)'s form (the block pattern of a cube element in the Walsh basis); d_x (float,
 * reference element order, x fastest), d_u and d_Ku (double, ndof) are device pointers; stream is a cudaStream_t as void*
 * (NULL: the legacy default stream).  The element moduli of the call live in a fixed
 * device array of TPO_STATIC_MAX_ELEMS doubles (8 MiB, held by every device that loads
 * the library until the process exits): larger grids return TPO_BAD_ARG.  The first
 * call on a device does its one-time set-up (scratch address, kernel shared-memory
 * limit) with that device current; make it before any stream capture.  There is one
 * scratch array per device, shared by every call, so calls on one device must not
 * overlap on the GPU (two streams or two host threads race on it). */
#define TPO_STATIC_MAX_ELEMS 1048576
tpo_status tpo_apply_static_dev(int32_t nelx, int32_t nely, int32_t nelz, const double *Ke,
                                const float *d_x, double penal, double E0, double Emin,
                                const double *d_u, double *d_Ku, void *stream);

#ifdef __cplusplus
}
#endif
#endif
