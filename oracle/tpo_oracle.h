/*
 * tpo_oracle.h -- CPU restatement of the reference's 3D SIMP finite-element path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA product
 * (libtpo.so) is compared against.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.  The product never links or calls it.
 *
 * Every function restates one routine of Jozo132/TopologyOptimization and cites the
 * file:line it follows.  Arithmetic is plain IEEE double evaluated left to right with
 * no fused multiply-add (build with -ffp-contract=off), which is what WebAssembly f64
 * and JavaScript numbers do.  Where the reference stores into a Float32Array the
 * oracle stores into float at the same point, so rounding happens where it does.
 *
 * Parity pinning: the reference cannot run in this container (no JavaScript or WASM
 * runtime), so this restatement is pinned by the reference's own known-answer tests
 * (tests/test-wasm-applyA.js, tests/test-wasm-mgpcg.js, tests/test-fea-benchmarks.js
 * scenarios and properties) and by an independent scipy sparse assembly + direct solve.
 */
#ifndef TPO_ORACLE_H
#define TPO_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- element and mesh ---------------------------------------------------- */
void orc_lk(double nu, double *Ke576);
void orc_edofs3d(int nelx, int nely, int nelz, int32_t *edofs);
/* position: 0 left, 1 right, 2 bottom, 3 top, 4 bottom-corners.
 * dofs bitmask: 1=x 2=y 4=z (7 = 'all').  Sets fixed[dof]=1. Returns count pushed. */
int orc_fixed_dofs(int nelx, int nely, int nelz, int position, int dofs, uint8_t *fixed);
/* preserved element mask of getConstraintElements (same position codes). */
void orc_constraint_elements(int nelx, int nely, int nelz, int position, uint8_t *mask);

/* ---- linear algebra kernels (assembly/index.ts) --------------------------- */
void orc_apply_a(const double *Ke, const int32_t *edofs, int edofSize, const double *evals,
                 const int32_t *active, int activeCount, const double *p, double *Ap, int ndof);
void orc_dense_matvec(const double *K, const double *p, double *Ap, int n);
int orc_ebe_pcg(const double *dens, const double *Ke, const int32_t *edofs, const double *F,
                double *U, const int32_t *freedofs, int nel, int edofSize, int ndof, int nfree,
                double Emin, double E0, double penal, int maxIter, double tol);

/* ---- geometric multigrid (js/optimizer-worker-3d.js MGPrecond3D + WASM core) - */
typedef struct orc_mg orc_mg;
typedef struct {
    int max_levels;        /* MG_MAX_LEVELS = 6 */
    int galerkin_max_ndof; /* GALERKIN_MAX_NDOF = 3000 */
    int nu1, nu2;          /* 2, 2 */
    double omega;          /* 0.5 */
    int coarse_iters;      /* 30 */
    int coarse_direct;     /* 0: reference sweeps; 1: Cholesky solve at the coarsest level */
    int coarse_moduli;     /* 0: reference (mean of raw child E, x2); 1: mean of active child E, x2 */
    int safe_omega;        /* 0: reference omega on every level; 1: min(omega, 1.9/bound) per level */
} orc_mg_opts;
void orc_mg_default_opts(orc_mg_opts *o);
orc_mg *orc_mg_create(int nelx, int nely, int nelz, const double *Ke, const uint8_t *fixedMask,
                      const orc_mg_opts *opts);
void orc_mg_destroy(orc_mg *mg);
int orc_mg_num_levels(const orc_mg *mg);
/* dims[8] = nelx, nely, nelz, ndof, nfree, activeCount, hasDense, nel */
void orc_mg_level_info(const orc_mg *mg, int li, int *dims);
void orc_mg_level_arrays(const orc_mg *mg, int li, double *evals, double *invDiag,
                         double *denseK /* may be NULL */);
void orc_mg_update(orc_mg *mg, const float *xFine, double penal, double E0, double Emin);
void orc_mg_apply_level(orc_mg *mg, int li, const double *p, double *Ap);
void orc_mg_set_spring(orc_mg *mg, long long dof, double k);
void orc_mg_vcycle(orc_mg *mg, const double *b, double *x); /* x is in/out on level 0 */
int orc_mgpcg(orc_mg *mg, const double *F, double *U, int maxIter, double tol); /* ebeMGPCG */
/* JS full-space PCG of FE() (:4189-4371). precond 0 = Jacobi, 1 = MG.  U in/out (warm). */
int orc_fe_pcg(orc_mg *mg, int precond, const double *F, double *U, int maxIter, double tol);

/* ---- KSP CG with the reference's "BDDC" preconditioner ------------------- */
/* Subdomains per axis of KSPSolver._buildSubdomains (js/optimizer-worker-3d.js:1141-1160). */
void orc_bddc_partition(int nelx, int nely, int nelz, int ns[3]);
/* _solveWithWasmKSP_BDDC + ebeKSP_BDDC (assembly/index.ts:1204-1517): cold start, E by
 * Math.pow, smootherIters local/global Jacobi steps per application (the worker's 3).
 * Returns the reference's iteration count (maxIter when not converged). */
int orc_ksp_bddc(int nelx, int nely, int nelz, const double *Ke, const float *x, double penal, double E0,
                 double Emin, const uint8_t *fixed, const double *F, double *U, int maxIter, double tol,
                 int smootherIters);

/* ---- SIMP pieces -------------------------------------------------------- */
void orc_element_energy(const double *Ke, int nelx, int nely, int nelz, const double *U,
                        float *energy);
void orc_element_energies_f32(const float *U, const float *KE, const int32_t *edofs, int nel, int es,
                              float *energies); /* GPUCompute's WGSL kernel */
void orc_stress(const float *xPhys, const float *energy, int n, double penal, double E0, double Emin,
                float *stress, double *max_stress); /* the volumetric stress field */
void orc_heaviside(const float *x, int n, double beta, float *xPhys);
void orc_sensitivity(const float *x, const float *xPhys, const float *energy, int n, double penal,
                     double E0, double beta, int useProjection, float *dc);
void orc_filter_hs(int nelx, int nely, int nelz, double rmin, float *Hs);
void orc_filter_sens(int nelx, int nely, int nelz, double rmin, const float *Hs, const float *x,
                     const float *dc, float *dcn);
void orc_density_filter(const double *dens, double *out, int nx, int ny, int nz, double radius);
void orc_oc(int nel, const float *x, double volfrac, const float *dc, const uint8_t *preserved,
            const uint8_t *voidm, float *xnew, double *lmid_out, int *nbisect_out);
void orc_oc_move(int nel, const float *x, double volfrac, const float *dc, const uint8_t *preserved,
                 const uint8_t *voidm, double move, float *xnew, double *lmid_out, int *nbisect_out);

/* ---- SIMP driver (optimize() :1605-2352, loop :2074-2301) ----------------- */
typedef struct {
    int nelx, nely, nelz;
    double volfrac, penal, rmin, E0, Emin, nu;
    int max_iter;
    double penal_start;     /* < 0: min(penal, 1.5) */
    int continuation_iters; /* < 0: max(20, floor(maxIter/3)) */
    int use_projection;
    double beta_max;
    int beta_interval;
    int solver;       /* 0 ebePCG, 1 ebeMGPCG, 2 JS PCG Jacobi, 3 JS PCG MG, 4 KSP with BDDC */
    int cg_max_iter;  /* the caller's cap: maxIter = min(nfree, cg_max_iter) */
    double cg_tol;    /* > 0 fixed tolerance, <= 0 the reference's schedule 1e-3 -> 1e-8 */
    int stop_on_change;
} orc_simp_cfg;
int orc_simp(const orc_simp_cfg *cfg, const float *F, const uint8_t *fixedMask,
             const uint8_t *preserved, const uint8_t *voidm, const orc_mg_opts *mgopts,
             double *c_hist, double *change_hist, int *cg_hist, float *x_out);

/* ---- the 2D worker (js/optimizer-worker.js) ------------------------------- */
void orc_lk2d(double nu, double *Ke64);
void orc_edofs2d(int nelx, int nely, int32_t *edofs);
void orc_filter_hs2d(int nelx, int nely, double rmin, float *Hs);
void orc_filter_sens2d(int nelx, int nely, double rmin, const float *Hs, const float *x, const float *dc, float *dcn);
typedef struct {
    int nelx, nely;
    double volfrac, penal, rmin, E0, Emin, nu;
    int max_iter;
    double penal_start;     /* < 0: min(penal, 1.5) */
    int continuation_iters; /* < 0: max(20, floor(maxIter/3)) */
    int use_projection;
    double beta_max;
    int beta_interval;
} orc_simp2d_cfg;
/* The loop of optimize() :580-730: tolerance max(1e-8, change * 1e-2), Jacobi-PCG solveCG
 * from zero with the absolute test, energies, sensitivities, 2D filter, OC, change.
 * F in a Float32Array (getLoadVector).  Returns the number of iterations. */
int orc_simp2d(const orc_simp2d_cfg *cfg, const float *F, const uint8_t *fixedMask, const uint8_t *preserved,
               const uint8_t *voidm, double *c_hist, double *change_hist, int *cg_hist, float *x_out);

#ifdef __cplusplus
}
#endif
#endif
