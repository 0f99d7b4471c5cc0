// Declarations of the non-apply kernels of libtpo (definitions in kernels.cu).
#pragma once
#include "common.cuh"

namespace tpo {

struct OCState {
    double l1, l2, lmid, last_lmid, sum;
    int done, nb;
    unsigned int counter;
};

// element stiffness
__global__ void k_lk(double nu, double *Ke);

// densities -> element moduli (internal z-fastest order) and thresholded copies
__global__ void k_evals_fine(const float *__restrict__ x_ref, Grid g, double penal, double E0,
                             double Emin, int intpow, double *__restrict__ E, double *__restrict__ Eact,
                             float *__restrict__ Eact32);
__global__ void k_evals_fine_f64(const double *__restrict__ x_ref, Grid g, double penal, double E0,
                                 double Emin, int intpow, double *__restrict__ E, double *__restrict__ Eact,
                                 float *__restrict__ Eact32);
__global__ void k_evals_avg(const double *__restrict__ Ef, Grid gf, Grid gc, double Emin,
                            double *__restrict__ Ec, double *__restrict__ Eact, float *__restrict__ Eact32);
__global__ void k_diag(const __grid_constant__ KeParam<double> ke, Grid g, const double *__restrict__ Eact,
                       const uint8_t *__restrict__ fixed, double *__restrict__ invD, float *__restrict__ invD32);

// dense coarse levels
__global__ void k_zero_d(double *a, long long n);
__global__ void k_galerkin_gather(const __grid_constant__ KeParam<double> ke, Grid gf, Grid gc,
                                  const double *__restrict__ EactF, double *__restrict__ Kc);
__global__ void k_galerkin_T(Grid gf, Grid gc, const double *__restrict__ Kf, double *__restrict__ T);
__global__ void k_galerkin_PtT(Grid gf, Grid gc, const double *__restrict__ T, double *__restrict__ Kc);
__global__ void k_dense_invdiag(const double *__restrict__ K, int n, const uint8_t *__restrict__ fixed,
                                double *__restrict__ invD, float *__restrict__ invD32);
// Gershgorin bound g = max over free rows with a positive diagonal of sum_j |K_ij| / K_ii
// (>= lambda_max(D^-1 K)); *womega = min(omega, 1.9 / g).  One block.
__global__ void k_dense_jacobi_bound(const double *__restrict__ K, int n, const uint8_t *__restrict__ fixed,
                                     double omega, double *__restrict__ womega);
__global__ void k_dense_matvec_seq(const double *__restrict__ K, int n, const double *__restrict__ p,
                                   double *__restrict__ Ap);
// coarsest level: explicit inverse
__global__ void k_coarse_prepare(const double *__restrict__ K, int n, const double *__restrict__ invD,
                                 double *__restrict__ A);
__global__ void k_gj_sweep(const double *__restrict__ A, double *__restrict__ B, int n, int k,
                           const double *__restrict__ invD);
__global__ void k_coarse_mask_inverse(const double *__restrict__ Ainv, int n, const double *__restrict__ invD,
                                      double *__restrict__ Kinv);

// PCG
__global__ void k_cg_setup(CGState *st, double tol, int maxIter, double eps);
__global__ void k_cg_init_r(const double *__restrict__ F, const double *__restrict__ Ku,
                            const uint8_t *__restrict__ fixed, double *__restrict__ U,
                            double *__restrict__ r, long long n, CGState *st, double *partials);
__global__ void k_cg_pz(const double *__restrict__ r, double *__restrict__ z, const double *__restrict__ invD,
                        const uint8_t *__restrict__ fixed, double *__restrict__ p, long long n, int jacobi,
                        CGState *st, double *partials);
__global__ void k_cg_update_mg(double *__restrict__ U, double *__restrict__ r, const double *__restrict__ p,
                               const double *__restrict__ Ap, long long n, CGState *st, double *partials);
__global__ void k_cg_rz(const double *__restrict__ r, double *__restrict__ z, const uint8_t *__restrict__ fixed,
                        long long n, CGState *st, double *partials);
__global__ void k_cg_update_jacobi(double *__restrict__ U, double *__restrict__ r, double *__restrict__ z,
                                   const double *__restrict__ p, const double *__restrict__ Ap,
                                   const double *__restrict__ invD, long long n, CGState *st, double *partials);
__global__ void k_cg_p(double *__restrict__ p, const double *__restrict__ z, long long n, const CGState *st);
__global__ void k_cg_alpha(const double *__restrict__ p, const double *__restrict__ Ap, long long n, CGState *st,
                           double *partials);
__global__ void k_mask_zero(double *__restrict__ a, const uint8_t *__restrict__ fixed, long long n);
__global__ void k_dot(const double *__restrict__ a, const double *__restrict__ b, long long n,
                      double *out, unsigned *counter, double *partials);

// general-edof apply (WASM ABI): per-element products, then a CSR gather per DOF
__global__ void k_elem_products(const double *__restrict__ Ke, int es, const int32_t *__restrict__ edofs,
                                const double *__restrict__ evals, const int32_t *__restrict__ elist,
                                int count, double thresh, const double *__restrict__ p,
                                double *__restrict__ y, const CGState *st);
__global__ void k_csr_gather(const int64_t *__restrict__ rowptr, const int64_t *__restrict__ cols,
                             const double *__restrict__ y, int ndof, double *__restrict__ out,
                             const uint8_t *__restrict__ fixed, const CGState *st);
__global__ void k_csr_apply(const double *__restrict__ Ke, int es, const int32_t *__restrict__ edofs,
                            const double *__restrict__ evals, double thresh, const double *__restrict__ p,
                            const int64_t *__restrict__ rowptr, const int64_t *__restrict__ cols, int ndof,
                            double *__restrict__ out, const uint8_t *__restrict__ fixed, const CGState *st);
__global__ void k_ebe_evals(const double *__restrict__ dens, int nel, double Emin, double E0, double penal,
                            double *__restrict__ E);
__global__ void k_diag_general(const double *__restrict__ Ke, int es, const int32_t *__restrict__ edofs,
                               const double *__restrict__ evals, int nel, double thresh,
                               double *__restrict__ ydiag);
__global__ void k_invdiag_general(const double *__restrict__ diag, const uint8_t *__restrict__ fixed,
                                  int n, double *__restrict__ invD);

// SIMP
__global__ void k_energy(const __grid_constant__ KeParam<double> ke, Grid g, const double *__restrict__ U,
                         float *__restrict__ energy);
__global__ void k_heaviside(const float *__restrict__ x, long long n, double beta, float *__restrict__ xp);
__global__ void k_sensitivity(const float *__restrict__ x, const float *__restrict__ xp, const float *__restrict__ en,
                              long long n, double penal, double E0, double beta, int useProj, int guard,
                              float *__restrict__ dc, double Emin, float *__restrict__ stress,
                              unsigned long long *__restrict__ max_stress_bits);
__global__ void k_filter_hs(Grid g, double rmin, float *__restrict__ Hs);
__global__ void k_filter_sens(Grid g, double rmin, const float *__restrict__ Hs, const float *__restrict__ x,
                              const float *__restrict__ dc, float *__restrict__ dcn);
__global__ void k_density_filter(Grid g, double radius, const double *__restrict__ in, double *__restrict__ out);
constexpr int kFilterTile = 8;     // elements per side of a tiled filter CTA
constexpr int kFilterMaxHalo = 4;  // largest stencil half-width of the tiled filters
__global__ void k_filter_sens_tiled(Grid g, double rmin, const float *__restrict__ Hs, const float *__restrict__ x,
                                    const float *__restrict__ dc, float *__restrict__ dcn);
__global__ void k_density_tiled(Grid g, double radius, int mode, const double *__restrict__ in,
                                double *__restrict__ out);
__global__ void k_oc_init(OCState *s);
// adjoint: dJ/dxPhys (reference order) and the density-filter transpose
__global__ void k_adjoint_sens(const __grid_constant__ KeParam<double> ke, Grid g, const double *__restrict__ xphys,
                               const double *__restrict__ U, const double *__restrict__ Lam, double penal, double E0,
                               double Emin, double *__restrict__ out);
__global__ void k_density_scale(Grid g, double radius, const double *__restrict__ gin, double *__restrict__ t);
__global__ void k_density_stencil(Grid g, double radius, const double *__restrict__ t, double *__restrict__ out);
__global__ void k_oc_step(const float *__restrict__ x, const float *__restrict__ dc,
                          const uint8_t *__restrict__ pres, const uint8_t *__restrict__ voidm, long long n,
                          double volfrac, double move, OCState *s, double *partials);
__global__ void k_oc_write(const float *__restrict__ x, const float *__restrict__ dc,
                           const uint8_t *__restrict__ pres, const uint8_t *__restrict__ voidm, long long n,
                           double move, const OCState *s, const float *__restrict__ xold,
                           float *__restrict__ xnew, unsigned long long *change_bits);

__global__ void k_energy_wgsl(const float *__restrict__ U, const float *__restrict__ KE,
                              const int32_t *__restrict__ edofs, int nel, int es, float *__restrict__ out);

// Structured subdomain partition of the reference's KSP "BDDC" preconditioner: block
// boundaries per axis (ns[a] blocks, b[k] .. b[k+1]).
constexpr int kBddcMaxBlocks = 64;
struct BddcPart {
    int ns[3];
    int bx[kBddcMaxBlocks + 1], by[kBddcMaxBlocks + 1], bz[kBddcMaxBlocks + 1];
};
__global__ void k_bddc_setup(const __grid_constant__ KeParam<double> ke, Grid g, const double *__restrict__ E,
                             const uint8_t *__restrict__ fixed, const __grid_constant__ BddcPart part,
                             double *__restrict__ S, uint8_t *__restrict__ W);
__global__ void k_bddc_local(const double *__restrict__ S, const uint8_t *__restrict__ W,
                             const double *__restrict__ r, double *__restrict__ z, long long n,
                             const CGState *__restrict__ st);

// the 2D worker's hot path
__global__ void k_evals_pow_f32(const float *__restrict__ x, int nel, double Emin, double E0, double penal,
                                double *__restrict__ E);
__global__ void k_energy_general(const double *__restrict__ Ke, int es, const int32_t *__restrict__ edofs,
                                 const double *__restrict__ U, int nel, float *__restrict__ energy);
__global__ void k_filter_hs2d(int nelx, int nely, double rmin, float *__restrict__ Hs);
__global__ void k_filter_sens2d(int nelx, int nely, double rmin, const float *__restrict__ Hs,
                                const float *__restrict__ x, const float *__restrict__ dc, float *__restrict__ dcn);

__global__ void k_cg_abs_tol(CGState *st, double tol);

}  // namespace tpo
