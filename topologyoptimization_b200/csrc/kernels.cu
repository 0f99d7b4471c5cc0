// Multigrid transfers, diagonals, dense coarse levels, PCG vector kernels and the
// element-energy kernel of libtpo.  Reference routines are cited per kernel
// (Jozo132/TopologyOptimization paths).
#include "kernels.cuh"

namespace tpo {

// _updateOperatorLevel step 1 (:753-771): E = Emin + x^p (E0 - Emin), active iff E > 1000 Emin.
// Reads densities in reference element order, writes z-fastest internal order.
__global__ void k_evals_fine(const float *__restrict__ x_ref, Grid g, double penal, double E0, double Emin,
                             int intpow, double *__restrict__ E, double *__restrict__ Eact,
                             float *__restrict__ Eact32) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.nel) return;
    const int ez = (int)(t % g.nelz);
    const long long r = t / g.nelz;
    const int ey = (int)(r % g.nely);
    const int ex = (int)(r / g.nely);
    const long long ref = ex + (long long)ey * g.nelx + (long long)ez * g.nelx * g.nely;
    const double x = (double)x_ref[ref];
    const double e = simp_modulus(x, penal, E0, Emin, intpow);
    E[t] = e;
    const double ea = e > Emin * 1000.0 ? e : 0.0;
    Eact[t] = ea;
    Eact32[t] = (float)ea;
}

// k_evals_fine from FP64 densities (the differentiable forward pass).
__global__ void k_evals_fine_f64(const double *__restrict__ x_ref, Grid g, double penal, double E0, double Emin,
                                 int intpow, double *__restrict__ E, double *__restrict__ Eact,
                                 float *__restrict__ Eact32) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.nel) return;
    const int ez = (int)(t % g.nelz);
    const long long r = t / g.nelz;
    const int ey = (int)(r % g.nely);
    const int ex = (int)(r / g.nely);
    const long long ref = ex + (long long)ey * g.nelx + (long long)ez * g.nelx * g.nely;
    const double e = simp_modulus(x_ref[ref], penal, E0, Emin, intpow);
    E[t] = e;
    const double ea = e > Emin * 1000.0 ? e : 0.0;
    Eact[t] = ea;
    Eact32[t] = (float)ea;
}

// _restrictEvalAvg (:702-739): coarse E = 2 * mean of the <= 8 children.
__global__ void k_evals_avg(const double *__restrict__ Ef, Grid gf, Grid gc, double Emin, double *__restrict__ Ec,
                            double *__restrict__ Eact, float *__restrict__ Eact32) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= gc.nel) return;
    const int cz = (int)(t % gc.nelz);
    const long long r = t / gc.nelz;
    const int cy = (int)(r % gc.nely);
    const int cx = (int)(r / gc.nely);
    double sum = 0.0;
    int count = 0;
    for (int dz = 0; dz < 2; dz++) {
        const int fz = 2 * cz + dz;
        if (fz >= gf.nelz) continue;
        for (int dy = 0; dy < 2; dy++) {
            const int fy = 2 * cy + dy;
            if (fy >= gf.nely) continue;
            for (int dx = 0; dx < 2; dx++) {
                const int fx = 2 * cx + dx;
                if (fx >= gf.nelx) continue;
                sum = __dadd_rn(sum, Ef[((long long)fx * gf.nely + fy) * gf.nelz + fz]);
                count++;
            }
        }
    }
    const double e = count > 0 ? __dmul_rn(sum / count, 2.0) : 0.0;
    Ec[t] = e;
    const double ea = e > Emin * 1000.0 ? e : 0.0;
    Eact[t] = ea;
    Eact32[t] = (float)ea;
}

// Jacobi diagonal (:773-795): diag = sum over active elements (ascending reference
// element index) of E_e * Ke_ii; invD = 1/diag on free DOFs with diag > 1e-30, else 0.
__global__ void k_diag(const __grid_constant__ KeParam<double> ke, Grid g, const double *__restrict__ Eact,
                       const uint8_t *__restrict__ fixed, double *__restrict__ invD, float *__restrict__ invD32) {
    const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= g.nnodes) return;
    const int z = (int)(n % g.nnz);
    const long long r = n / g.nnz;
    const int y = (int)(r % g.nny);
    const int x = (int)(r / g.nny);
    double dg[3] = {0.0, 0.0, 0.0};
    for (int az = 0; az < 2; az++) {
        const int ez = z - 1 + az;
        if (ez < 0 || ez >= g.nelz) continue;
        for (int ay = 0; ay < 2; ay++) {
            const int ey = y - 1 + ay;
            if (ey < 0 || ey >= g.nely) continue;
            for (int ax = 0; ax < 2; ax++) {
                const int ex = x - 1 + ax;
                if (ex < 0 || ex >= g.nelx) continue;
                const double E = Eact[((long long)ex * g.nely + ey) * g.nelz + ez];
                const int L = local_node(1 - ax, 1 - ay, 1 - az);
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int q = 3 * L + d;
                    dg[d] = __dadd_rn(dg[d], __dmul_rn(E, ke.v[q * 24 + q]));
                }
            }
        }
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const long long i = 3 * n + d;
        if (i == g.sdof) dg[d] += g.sk;
        const double v = (!fixed[i] && dg[d] > 1e-30) ? 1.0 / dg[d] : 0.0;
        invD[i] = v;
        invD32[i] = (float)v;
    }
}

// ---- dense Galerkin coarse levels (:628-699) --------------------------------------
// Damping of the dense levels under safe_omega: damped Jacobi x += w D^-1 (b - K x)
// converges (and keeps the symmetric V-cycle positive definite) iff w lambda_max(D^-1 K) < 2;
// the Gershgorin row bound g >= lambda_max gives the damping w = min(omega, 1.9 / g).
// Rows are summed in column order, as the oracle does.
__global__ void k_dense_jacobi_bound(const double *__restrict__ K, int n, const uint8_t *__restrict__ fixed,
                                     double omega, double *__restrict__ womega) {
    double g = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double d = K[(long long)i * n + i];
        if (fixed[i] || !(d > 1e-30)) continue;
        double s = 0.0;
        for (int j = 0; j < n; j++) s += fabs(K[(long long)i * n + j]);
        g = fmax(g, s / d);
    }
    for (int o = 16; o > 0; o >>= 1) g = fmax(g, __shfl_xor_sync(0xffffffffu, g, o));
    __shared__ double sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = g;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) g = fmax(g, sh[w]);
        g = fmax(g, sh[0]);
        *womega = g > 0.0 ? fmin(omega, 1.9 / g) : omega;
    }
}

__global__ void k_zero_d(double *a, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] = 0.0;
}

__device__ __forceinline__ int prolong_list(Grid gf, Grid gc, long long nf, int *cn, double *cw) {
    const int fz = (int)(nf % gf.nnz);
    const long long r = nf / gf.nnz;
    const int fy = (int)(r % gf.nny);
    const int fx = (int)(r / gf.nny);
    int cx[2], cy[2], cz[2];
    double wx[2], wy[2], wz[2];
    {
        const int c0 = min(fx >> 1, gc.nnx - 1), c1 = min(c0 + 1, gc.nnx - 1);
        const double t = (c0 != c1 && (fx & 1)) ? 0.5 : 0.0;
        cx[0] = c0; cx[1] = c1; wx[0] = 1 - t; wx[1] = t;
    }
    {
        const int c0 = min(fy >> 1, gc.nny - 1), c1 = min(c0 + 1, gc.nny - 1);
        const double t = (c0 != c1 && (fy & 1)) ? 0.5 : 0.0;
        cy[0] = c0; cy[1] = c1; wy[0] = 1 - t; wy[1] = t;
    }
    {
        const int c0 = min(fz >> 1, gc.nnz - 1), c1 = min(c0 + 1, gc.nnz - 1);
        const double t = (c0 != c1 && (fz & 1)) ? 0.5 : 0.0;
        cz[0] = c0; cz[1] = c1; wz[0] = 1 - t; wz[1] = t;
    }
    int cnt = 0;
    for (int dz = 0; dz < 2; dz++)
        for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++) {
                const double w = wx[dx] * wy[dy] * wz[dz];
                if (w > 0) {
                    cn[cnt] = (cx[dx] * gc.nny + cy[dy]) * gc.nnz + cz[dz];
                    cw[cnt] = w;
                    cnt++;
                }
            }
    return cnt;
}

// _assembleGalerkinFromMatrix, first product T = Kf P.  T[i][3c+d] sums Kf[i][3f+d] w(f,c)
// over the fine nodes f that interpolate from c, in ascending f (the order of the
// reference's dense k loop once its zero terms are dropped).
__global__ void k_galerkin_T(Grid gf, Grid gc, const double *__restrict__ Kf, double *__restrict__ T) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nF = gf.ndof, nC = gc.ndof;
    if (t >= nF * nC) return;
    const long long i = t / nC, j = t % nC;
    const long long cn = j / 3;
    const int d = (int)(j % 3);
    const int cz = (int)(cn % gc.nnz);
    const long long r = cn / gc.nnz;
    const int cy = (int)(r % gc.nny);
    const int cx = (int)(r / gc.nny);
    double s = 0.0;
    for (int fx = 2 * cx - 1; fx <= 2 * cx + 1; fx++) {
        if (fx < 0 || fx >= gf.nnx) continue;
        const double wx = w1d(fx, cx, gc.nnx);
        if (wx == 0.0) continue;
        for (int fy = 2 * cy - 1; fy <= 2 * cy + 1; fy++) {
            if (fy < 0 || fy >= gf.nny) continue;
            const double wy = w1d(fy, cy, gc.nny);
            if (wy == 0.0) continue;
            for (int fz = 2 * cz - 1; fz <= 2 * cz + 1; fz++) {
                if (fz < 0 || fz >= gf.nnz) continue;
                const double wz = w1d(fz, cz, gc.nnz);
                const double w = wx * wy * wz;
                if (!(w > 0.0)) continue;
                const long long nf = ((long long)fx * gf.nny + fy) * gf.nnz + fz;
                s = s + Kf[i * nF + 3 * nf + d] * w;
            }
        }
    }
    T[t] = s;
}

// Second product Kc = P^T T.
__global__ void k_galerkin_PtT(Grid gf, Grid gc, const double *__restrict__ T, double *__restrict__ Kc) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nC = gc.ndof;
    if (t >= nC * nC) return;
    const long long a = t / nC, b = t % nC;
    const long long cn = a / 3;
    const int d = (int)(a % 3);
    const int cz = (int)(cn % gc.nnz);
    const long long r = cn / gc.nnz;
    const int cy = (int)(r % gc.nny);
    const int cx = (int)(r / gc.nny);
    double s = 0.0;
    for (int fx = 2 * cx - 1; fx <= 2 * cx + 1; fx++) {
        if (fx < 0 || fx >= gf.nnx) continue;
        const double wx = w1d(fx, cx, gc.nnx);
        if (wx == 0.0) continue;
        for (int fy = 2 * cy - 1; fy <= 2 * cy + 1; fy++) {
            if (fy < 0 || fy >= gf.nny) continue;
            const double wy = w1d(fy, cy, gc.nny);
            if (wy == 0.0) continue;
            for (int fz = 2 * cz - 1; fz <= 2 * cz + 1; fz++) {
                if (fz < 0 || fz >= gf.nnz) continue;
                const double wz = w1d(fz, cz, gc.nnz);
                const double w = wx * wy * wz;
                if (!(w > 0.0)) continue;
                const long long nf = ((long long)fx * gf.nny + fy) * gf.nnz + fz;
                s = s + w * T[(3 * nf + d) * nC + b];
            }
        }
    }
    Kc[t] = s;
}

// _diagFromDense (:742-751)
__global__ void k_dense_invdiag(const double *__restrict__ K, int n, const uint8_t *__restrict__ fixed,
                                double *__restrict__ invD, float *__restrict__ invD32) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = K[(long long)i * n + i];
    const double v = (!fixed[i] && d > 1e-30) ? 1.0 / d : 0.0;
    invD[i] = v;
    invD32[i] = (float)v;
}

// ---- coarsest level: explicit inverse of the dense operator -------------------------
// The operator restricted to its free, non-singular DOFs: rows/columns whose inverse
// diagonal is 0 (fixed DOFs, DOFs without active elements) become identity rows.
__global__ void k_coarse_prepare(const double *__restrict__ K, int n, const double *__restrict__ invD,
                                 double *__restrict__ A) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n * n) return;
    const int i = (int)(t / n), j = (int)(t % n);
    const bool ci = invD[i] == 0.0, cj = invD[j] == 0.0;
    A[t] = (ci || cj) ? (i == j ? 1.0 : 0.0) : K[t];
}

// One Gauss-Jordan sweep of pivot k, A -> B (both n x n, row-major): after sweeping every
// pivot of a symmetric positive definite A in turn, the matrix holds A^-1.  The pivot
// a_kk at step k is the Schur complement of the pivots swept before it, i.e. the d of a
// Cholesky factorisation; a pivot at or below 1e-10 of the row's diagonal (1 / invD, or 1
// on a decoupled row) is a singular direction up to rounding (a floating island of active
// elements) and is replaced by 1, the same modification of A as the oracle's Cholesky
// makes.  Reading A and writing B keeps the pivot row and column intact while they are read.
__global__ void k_gj_sweep(const double *__restrict__ A, double *__restrict__ B, int n, int k,
                           const double *__restrict__ invD) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n * n) return;
    const int i = (int)(t / n), j = (int)(t - (long long)i * n);
    const double dk = invD[k] == 0.0 ? 1.0 : 1.0 / invD[k];
    double p = A[(long long)k * n + k];
    if (!(p > 1e-10 * dk)) p = 1.0;
    const double ip = 1.0 / p;
    const double aik = A[(long long)i * n + k], akj = A[(long long)k * n + j];
    double v;
    if (i == k) v = (j == k) ? ip : akj * ip;
    else if (j == k) v = -aik * ip;
    else v = A[t] - aik * (akj * ip);
    B[t] = v;
}

// Kinv = Ainv with zero rows and columns on DOFs whose invD is 0 (their coarse solution is 0).
__global__ void k_coarse_mask_inverse(const double *__restrict__ Ainv, int n, const double *__restrict__ invD,
                                      double *__restrict__ Kinv) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n * n) return;
    const int i = (int)(t / n), j = (int)(t - (long long)i * n);
    Kinv[t] = (invD[i] == 0.0 || invD[j] == 0.0) ? 0.0 : Ainv[t];
}

// ---- PCG (ebePCG assembly/index.ts:504-733, ebeMGPCG :1076-1193, FE :4189-4371) -----
__global__ void k_cg_setup(CGState *st, double tol, int maxIter, double eps) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    st += zr;
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    st->rz = st->rz_new = st->pAp = st->alpha = st->beta = st->rr = st->r0 = 0.0;
    st->tolSq = tol;  // squared in k_cg_init_r once ||r0|| is known
    st->eps = eps;
    st->it = 0;
    st->done = 0;
    st->iters = 0;
    st->converged = 0;
    st->maxIter = maxIter;
    st->nonfinite = 0;
    st->rr32 = st->maxr2 = st->delta2 = 0.0;  // not the mixed recurrence
    st->do_update = st->n_updates = 0;
    for (int k = 0; k < 8; k++) st->counters[k] = 0u;
}

// An absolute stopping test ||r||^2 < tol^2 in place of the relative one (the 2D worker's
// solveCG, js/optimizer-worker.js:1841-1845); runs between k_cg_init_r and k_cg_pz.
__global__ void k_cg_abs_tol(CGState *st, double tol) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    st->tolSq = tol * tol;
}

// r = F - K U on free DOFs (Ku == null: cold start, U = 0), 0 on fixed; ||r0||^2.
__global__ void k_cg_init_r(const double *__restrict__ F, const double *__restrict__ Ku,
                            const uint8_t *__restrict__ fixed, double *__restrict__ U, double *__restrict__ r,
                            long long n, CGState *st, double *partials) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    F += zr * n;
    if (Ku) Ku += zr * n;
    U += zr * n;
    r += zr * n;
    st += zr;
    double v[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double ri;
        if (Ku) {
            ri = fixed[i] ? 0.0 : F[i] - Ku[i];
        } else {
            U[i] = 0.0;
            ri = fixed[i] ? 0.0 : F[i];
        }
        r[i] = ri;
        v[0] += ri * ri;
    }
    __shared__ double sh[32];
    double tot[1];
    if (grid_sum<1>(v, partials, &st->counters[0], sh, tot) && threadIdx.x == 0) {
        st->r0 = tot[0];
        st->rr = tot[0];
        const double tol = st->tolSq;
        st->tolSq = tol * tol * (tot[0] > 1e-30 ? tot[0] : 1e-30);
        if (!isfinite(tot[0])) {
            st->nonfinite = 1;
            st->done = 1;
        }
    }
}

// z = invD r (jacobi) or the preconditioned z, zeroed on fixed DOFs; p = z; rz = r.z.
// Then the reference's first convergence test (rr < tolSq -> 0 iterations).
__global__ void k_cg_pz(const double *__restrict__ r, double *__restrict__ z, const double *__restrict__ invD,
                        const uint8_t *__restrict__ fixed, double *__restrict__ p, long long n, int jacobi,
                        CGState *st, double *partials) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    r += zr * n;
    z += zr * n;
    p += zr * n;
    st += zr;
    if (st->done) return;
    double v[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double ri = r[i];
        double zi = jacobi ? invD[i] * ri : z[i];
        if (fixed[i]) zi = 0.0;
        z[i] = zi;
        p[i] = zi;
        v[0] += ri * zi;
    }
    __shared__ double sh[32];
    double tot[1];
    if (grid_sum<1>(v, partials, &st->counters[1], sh, tot) && threadIdx.x == 0) {
        st->rz = tot[0];
        if (st->rr < st->tolSq) {
            st->done = 1;
            st->converged = 1;
            st->iters = 0;
        } else if (st->maxIter <= 0) {
            st->done = 1;
            st->iters = 0;
        }
    }
}

// U += alpha p; r -= alpha Ap; rr = r.r (MG variant: z comes from the V-cycle next).
__global__ void k_cg_update_mg(double *__restrict__ U, double *__restrict__ r, const double *__restrict__ p,
                               const double *__restrict__ Ap, long long n, CGState *st, double *partials) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    U += zr * n;
    r += zr * n;
    p += zr * n;
    Ap += zr * n;
    st += zr;
    if (st->done) return;
    const double alpha = st->alpha;
    double v[1] = {0.0};
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
    const bool vec = aligned_to(16, U, r, p, Ap);
    const long long nv = n / 2;
    for (long long i = t0; i < nv; i += stride) {  // pairs of DOFs
        Pair<double> u = ld_pair(U, i, vec), rr = ld_pair(r, i, vec);
        const Pair<double> pp = ld_pair(p, i, vec), ap = ld_pair(Ap, i, vec);
        u.x = u.x + alpha * pp.x;
        u.y = u.y + alpha * pp.y;
        rr.x = rr.x - alpha * ap.x;
        rr.y = rr.y - alpha * ap.y;
        st_pair(U, i, u, vec);
        st_pair(r, i, rr, vec);
        v[0] += rr.x * rr.x;
        v[0] += rr.y * rr.y;
    }
    for (long long i = 2 * nv + t0; i < n; i += stride) {
        U[i] = U[i] + alpha * p[i];
        const double ri = r[i] - alpha * Ap[i];
        r[i] = ri;
        v[0] += ri * ri;
    }
    __shared__ double sh[32];
    double tot[1];
    if (grid_sum<1>(v, partials, &st->counters[2], sh, tot) && threadIdx.x == 0) {
        st->rr = tot[0];
        cg_decide(st);
    }
}

// z zeroed on fixed DOFs; rz_new = r.z; beta.
__global__ void k_cg_rz(const double *__restrict__ r, double *__restrict__ z, const uint8_t *__restrict__ fixed,
                        long long n, CGState *st, double *partials) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    r += zr * n;
    z += zr * n;
    st += zr;
    if (st->done) return;
    double v[1] = {0.0};
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
    const bool vec = aligned_to(16, r, z);
    const long long nv = n / 2;
    for (long long i = t0; i < nv; i += stride) {  // pairs of DOFs
        const Pair<double> rr = ld_pair(r, i, vec);
        Pair<double> zz = ld_pair(z, i, vec);
        const uint8_t f0 = fixed[2 * i], f1 = fixed[2 * i + 1];
        if (f0 || f1) {
            if (f0) zz.x = 0.0;
            if (f1) zz.y = 0.0;
            st_pair(z, i, zz, vec);
        }
        v[0] += rr.x * zz.x;
        v[0] += rr.y * zz.y;
    }
    for (long long i = 2 * nv + t0; i < n; i += stride) {
        double zi = z[i];
        if (fixed[i]) {
            zi = 0.0;
            z[i] = 0.0;
        }
        v[0] += r[i] * zi;
    }
    __shared__ double sh[32];
    double tot[1];
    if (grid_sum<1>(v, partials, &st->counters[3], sh, tot) && threadIdx.x == 0) {
        st->rz_new = tot[0];
        if (st->eps > 0.0) st->beta = tot[0] / (st->rz + st->eps);
        else st->beta = st->rz > 0.0 ? tot[0] / st->rz : 0.0;
        st->rz = tot[0];
    }
}

// Jacobi variant: U += alpha p; r -= alpha Ap; z = invD r; rz_new and rr in one pass.
__global__ void k_cg_update_jacobi(double *__restrict__ U, double *__restrict__ r, double *__restrict__ z,
                                   const double *__restrict__ p, const double *__restrict__ Ap,
                                   const double *__restrict__ invD, long long n, CGState *st, double *partials) {
    if (st->done) return;
    const double alpha = st->alpha;
    double v[2] = {0.0, 0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double ri = r[i] - alpha * Ap[i];
        const double zi = invD[i] * ri;
        U[i] = U[i] + alpha * p[i];
        r[i] = ri;
        z[i] = zi;
        v[0] += ri * zi;
        v[1] += ri * ri;
    }
    __shared__ double sh[64];
    double tot[2];
    if (grid_sum<2>(v, partials, &st->counters[2], sh, tot) && threadIdx.x == 0) {
        st->rz_new = tot[0];
        if (st->eps > 0.0) st->beta = tot[0] / (st->rz + st->eps);
        else st->beta = st->rz > 0.0 ? tot[0] / st->rz : 0.0;
        st->rz = tot[0];
        st->rr = tot[1];
        cg_decide(st);
    }
}

__global__ void k_cg_p(double *__restrict__ p, const double *__restrict__ z, long long n, const CGState *st) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    p += zr * n;
    z += zr * n;
    st += zr;
    if (st->done) return;
    const double beta = st->beta;
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
    const bool vec = aligned_to(16, p, z);
    const long long nv = n / 2;
    for (long long i = t0; i < nv; i += stride) {  // pairs of DOFs
        Pair<double> pp = ld_pair(p, i, vec);
        const Pair<double> zz = ld_pair(z, i, vec);
        pp.x = zz.x + beta * pp.x;
        pp.y = zz.y + beta * pp.y;
        st_pair(p, i, pp, vec);
    }
    for (long long i = 2 * nv + t0; i < n; i += stride) p[i] = z[i] + beta * p[i];
}

// alpha = rz / (p.Ap + eps) for operators without a fused epilogue (general-edof path).
__global__ void k_cg_alpha(const double *__restrict__ p, const double *__restrict__ Ap, long long n, CGState *st,
                           double *partials) {
    if (st->done) return;
    double v[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[0] += p[i] * Ap[i];
    __shared__ double sh[32];
    double tot[1];
    if (grid_sum<1>(v, partials, &st->counters[4], sh, tot) && threadIdx.x == 0) {
        st->pAp = tot[0];
        if (st->eps > 0.0) {
            st->alpha = st->rz / (tot[0] + st->eps);
        } else if (tot[0] > 0.0) {
            st->alpha = st->rz / tot[0];
        } else {
            st->alpha = 0.0;
            st->done = 1;
            st->iters = st->it;
        }
    }
}

__global__ void k_mask_zero(double *__restrict__ a, const uint8_t *__restrict__ fixed, long long n) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    a += zr * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (fixed[i]) a[i] = 0.0;
}

__global__ void k_dot(const double *__restrict__ a, const double *__restrict__ b, long long n, double *out,
                      unsigned *counter, double *partials) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    a += zr * n;
    b += zr * n;
    out += zr;
    counter += zr;
    double v[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[0] += a[i] * b[i];
    __shared__ double sh[32];
    double tot[1];
    if (grid_sum<1>(v, partials, counter, sh, tot) && threadIdx.x == 0) *out = tot[0];
}

// ---- element energy (:2163-2173, unit Ke, every element) ---------------------------
// One thread per element in z-fastest order (coalesced node reads); the float result is
// written at the reference element index.
__global__ void k_energy(const __grid_constant__ KeParam<double> ke, Grid g, const double *__restrict__ U,
                         float *__restrict__ energy) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.nel) return;
    const int ez = (int)(t % g.nelz);
    const long long r = t / g.nelz;
    const int ey = (int)(r % g.nely);
    const int ex = (int)(r / g.nely);
    double u[24];
#pragma unroll
    for (int b = 0; b < 8; b++) {
        const int ox = (b == 1 || b == 2 || b == 5 || b == 6);
        const int oy = (b == 2 || b == 3 || b == 6 || b == 7);
        const int oz = (b >= 4);
        const long long nd = ((long long)(ex + ox) * g.nny + (ey + oy)) * g.nnz + (ez + oz);
#pragma unroll
        for (int q = 0; q < 3; q++) u[b * 3 + q] = U[3 * nd + q];
    }
    double en = 0.0;
#pragma unroll
    for (int i = 0; i < 24; i++) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < 24; j++) s = fma(ke.v[i * 24 + j], u[j], s);
        en = fma(u[i], s, en);
    }
    energy[ex + (long long)ey * g.nelx + (long long)ez * g.nelx * g.nely] = (float)en;
}

// ---- Heaviside projection and sensitivity (:3500-3509, :2175-2192) ------------------
__global__ void k_heaviside(const float *__restrict__ x, long long n, double beta, float *__restrict__ xp) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double eta = 0.5;
    const double tb = tanh(beta * eta), tb1 = tanh(beta * (1 - eta));
    xp[i] = (float)((tb + tanh(beta * ((double)x[i] - eta))) / (tb + tb1));
}

__global__ void k_sensitivity(const float *__restrict__ x, const float *__restrict__ xp, const float *__restrict__ en,
                              long long n, double penal, double E0, double beta, int useProj, int guard,
                              float *__restrict__ dc, double Emin, float *__restrict__ stress,
                              unsigned long long *__restrict__ max_stress_bits) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (stress) {
        // the volumetric stress field of the loop (js/optimizer-worker-3d.js:2180-2184):
        // (Emin + xPhys^p (E0 - Emin)) * energy by Math.pow, two roundings, stored as float;
        // its maximum over the elements starts at 0.  Positive doubles order as their bit
        // patterns, so the maximum is an integer maximum: per warp by shuffles, per block in
        // shared memory, one atomic per block.
        unsigned long long mb = 0;
        if (e < n) {
            const double stiff = __dadd_rn(Emin, __dmul_rn(pow((double)xp[e], penal), E0 - Emin));
            const double sv = __dmul_rn(stiff, (double)en[e]);
            stress[e] = (float)sv;
            if (sv > 0.0) mb = (unsigned long long)__double_as_longlong(sv);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long v = __shfl_down_sync(0xffffffffu, mb, o);
            mb = v > mb ? v : mb;
        }
        __shared__ unsigned long long wmax[32];
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0) wmax[w] = mb;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long m = 0;
            for (int i = 0; i < (int)(blockDim.x >> 5); i++) m = wmax[i] > m ? wmax[i] : m;
            if (m) atomicMax(max_stress_bits, m);
        }
    }
    if (e >= n) return;
    const double hden = 2 * tanh(beta * 0.5);
    // guard: the element energy u_e^T Ke u_e is >= 0 for the positive semidefinite Ke; a
    // rounding-negative value would make dc > 0 and sqrt(-dc/lambda) NaN in the OC update
    const double ene = guard ? fmax((double)en[e], 0.0) : (double)en[e];
    const double dcp = -penal * pow((double)xp[e], penal - 1) * E0 * ene;
    const double th = tanh(beta * ((double)x[e] - 0.5));
    const double dpdx = useProj ? beta * (1 - th * th) / hden : 1.0;
    dc[e] = (float)(dcp * dpdx);
}

}  // namespace tpo

namespace tpo {

// ---- adjoint sensitivities ---------------------------------------------------------------
// dJ/dxPhys_e = -p xPhys_e^(p-1) (E0 - Emin) lambda_e^T Ke u_e for J = l.u with K lambda = l
// (lambda = u for the compliance J = F.u).  Output in reference element order.
__global__ void k_adjoint_sens(const __grid_constant__ KeParam<double> ke, Grid g, const double *__restrict__ xphys,
                               const double *__restrict__ U, const double *__restrict__ Lam, double penal, double E0,
                               double Emin, double *__restrict__ out) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.nel) return;
    const int ez = (int)(t % g.nelz);
    const long long r = t / g.nelz;
    const int ey = (int)(r % g.nely);
    const int ex = (int)(r / g.nely);
    double u[24], lam[24];
#pragma unroll
    for (int b = 0; b < 8; b++) {
        const int ox = (b == 1 || b == 2 || b == 5 || b == 6);
        const int oy = (b == 2 || b == 3 || b == 6 || b == 7);
        const int oz = (b >= 4);
        const long long nd = ((long long)(ex + ox) * g.nny + (ey + oy)) * g.nnz + (ez + oz);
#pragma unroll
        for (int q = 0; q < 3; q++) {
            u[b * 3 + q] = U[3 * nd + q];
            lam[b * 3 + q] = Lam[3 * nd + q];
        }
    }
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < 24; i++) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < 24; j++) s = fma(ke.v[i * 24 + j], u[j], s);
        m = fma(lam[i], s, m);
    }
    const long long ref = ex + (long long)ey * g.nelx + (long long)ez * g.nelx * g.nely;
    out[ref] = -penal * pow(xphys[ref], penal - 1.0) * (E0 - Emin) * m;
}

// Transpose of the density filter xPhys_e = sum_k w_ek x_k / sum_k w_ek (w = r - dist over
// dist^2 <= r^2, the stencil of k_density_filter; the neighbourhood relation is symmetric):
// step 1 t_e = g_e / sum_k w_ek, step 2 out_k = sum_e w_ek t_e.
__global__ void k_density_scale(Grid g, double radius, const double *__restrict__ gin, double *__restrict__ t) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= g.nel) return;
    const int ex = (int)(e % g.nelx);
    const long long r = e / g.nelx;
    const int ey = (int)(r % g.nely);
    const int ez = (int)(r / g.nely);
    const int R = (int)ceil(radius);
    const double r2 = radius * radius;
    double sw = 0.0;
    for (int kz = max(0, ez - R); kz <= min(g.nelz - 1, ez + R); kz++)
        for (int ky = max(0, ey - R); ky <= min(g.nely - 1, ey + R); ky++)
            for (int kx = max(0, ex - R); kx <= min(g.nelx - 1, ex + R); kx++) {
                const double dx = ex - kx, dy = ey - ky, dz = ez - kz;
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 <= r2) sw += radius - sqrt(d2);
            }
    t[e] = gin[e] / sw;
}
__global__ void k_density_stencil(Grid g, double radius, const double *__restrict__ t, double *__restrict__ out) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= g.nel) return;
    const int ex = (int)(e % g.nelx);
    const long long r = e / g.nelx;
    const int ey = (int)(r % g.nely);
    const int ez = (int)(r / g.nely);
    const int R = (int)ceil(radius);
    const double r2 = radius * radius;
    double sum = 0.0;
    for (int kz = max(0, ez - R); kz <= min(g.nelz - 1, ez + R); kz++)
        for (int ky = max(0, ey - R); ky <= min(g.nely - 1, ey + R); ky++)
            for (int kx = max(0, ex - R); kx <= min(g.nelx - 1, ex + R); kx++) {
                const double dx = ex - kx, dy = ey - ky, dz = ez - kz;
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 <= r2) sum += (radius - sqrt(d2)) * __ldg(&t[kx + (long long)ky * g.nelx + (long long)kz * g.nelx * g.nely]);
            }
    out[e] = sum;
}

// ---- the reference's "BDDC" preconditioner (KSPSolver, js/optimizer-worker-3d.js:1141-1231;
// bddcApply, assembly/index.ts:1264-1353) --------------------------------------------------
// Subdomains are the blocks [b[k], b[k+1]) of a structured partition per axis, numbered
// (sz, sy, sx) with sx fastest, empty blocks dropped.  A node at coordinate v lies in
// block k of an axis when b[k] <= v <= b[k+1] (one or two blocks per axis).
__device__ __forceinline__ int bddc_blocks(const int *b, int nb, int v, int (&out)[2]) {
    int n = 0;
    for (int k = 0; k < nb && n < 2; k++)
        if (b[k + 1] > b[k] && b[k] <= v && v <= b[k + 1]) out[n++] = k;
    return n;
}

// Per DOF: S = sum over the node's subdomains (in subdomain order) of the local inverse
// diagonal (1 / sum of E_e Ke_ii over the subdomain's elements at the node, every element
// with E >= 1e-30; 0 on fixed DOFs or a diagonal <= 1e-30), W = the number of those
// subdomains.  Step 1 of bddcApply is then z = S r / W.
__global__ void k_bddc_setup(const __grid_constant__ KeParam<double> ke, Grid g, const double *__restrict__ E,
                             const uint8_t *__restrict__ fixed, const __grid_constant__ BddcPart part,
                             double *__restrict__ S, uint8_t *__restrict__ W) {
    const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= g.nnodes) return;
    int x, y, z;
    node_xyz(g, n, x, y, z);
    int bx[2], by[2], bz[2];
    const int cx = bddc_blocks(part.bx, part.ns[0], x, bx);
    const int cy = bddc_blocks(part.by, part.ns[1], y, by);
    const int cz = bddc_blocks(part.bz, part.ns[2], z, bz);
    double s[3] = {0.0, 0.0, 0.0};
    for (int iz = 0; iz < cz; iz++)
        for (int iy = 0; iy < cy; iy++)
            for (int ix = 0; ix < cx; ix++) {
                double ld[3] = {0.0, 0.0, 0.0};
                for (int ez = max(z - 1, part.bz[bz[iz]]); ez <= min(z, part.bz[bz[iz] + 1] - 1); ez++)
                    for (int ey = max(y - 1, part.by[by[iy]]); ey <= min(y, part.by[by[iy] + 1] - 1); ey++)
                        for (int ex = max(x - 1, part.bx[bx[ix]]); ex <= min(x, part.bx[bx[ix] + 1] - 1); ex++) {
                            const double Ee = E[((long long)ex * g.nely + ey) * g.nelz + ez];
                            if (Ee < 1e-30) continue;
                            const int L = local_node(x - ex, y - ey, z - ez);
#pragma unroll
                            for (int d = 0; d < 3; d++)
                                ld[d] = __dadd_rn(ld[d], __dmul_rn(Ee, ke.v[(3 * L + d) * 24 + 3 * L + d]));
                        }
#pragma unroll
                for (int d = 0; d < 3; d++)
                    s[d] = __dadd_rn(s[d], (!fixed[3 * n + d] && ld[d] > 1e-30) ? 1.0 / ld[d] : 0.0);
            }
#pragma unroll
    for (int d = 0; d < 3; d++) {
        S[3 * n + d] = s[d];
        W[3 * n + d] = (uint8_t)(cx * cy * cz);
    }
}

// z = S r / W (grid z: right-hand sides)
__global__ void k_bddc_local(const double *__restrict__ S, const uint8_t *__restrict__ W,
                             const double *__restrict__ r, double *__restrict__ z, long long n,
                             const CGState *__restrict__ st) {
    if (blockIdx.z) {
        r += blockIdx.z * n;
        z += blockIdx.z * n;
        if (st) st += blockIdx.z;
    }
    if (st && st->done) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double v = S[i] * r[i];
        z[i] = W[i] ? v / (double)W[i] : v;
    }
}

}  // namespace tpo
