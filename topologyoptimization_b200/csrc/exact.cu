// Kernels whose arithmetic must follow the reference operation by operation.  This file
// is compiled with --fmad=false so that a*b+c stays two rounded operations, as in
// WebAssembly f64 and JavaScript.  Sums run in the reference's order.
#include "kernels.cuh"

namespace tpo {

// JavaScript Math.max / Math.min: NaN propagates; +0 wins max, -0 wins min.
__device__ __forceinline__ double js_max(double a, double b) {
    if (a != a || b != b) return __longlong_as_double(0x7ff8000000000000LL);
    if (a == b) return signbit(a) ? b : a;
    return a > b ? a : b;
}
__device__ __forceinline__ double js_min(double a, double b) {
    if (a != a || b != b) return __longlong_as_double(0x7ff8000000000000LL);
    if (a == b) return signbit(a) ? a : b;
    return a < b ? a : b;
}

// lk() (js/optimizer-worker-3d.js:3404-3491): one thread per entry (m, n), same
// sequence of operations as the reference's Gauss loop.
__global__ void k_lk(double nu, double *Ke) {
    const int t = threadIdx.x;
    if (t >= 576) return;
    const int m = t / 24, n = t % 24;
    const double E = 1.0;
    double C[6][6];
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) C[a][b] = 0.0;
    const double fact = E / ((1 + nu) * (1 - 2 * nu));
    C[0][0] = fact * (1 - nu); C[0][1] = fact * nu; C[0][2] = fact * nu;
    C[1][0] = fact * nu; C[1][1] = fact * (1 - nu); C[1][2] = fact * nu;
    C[2][0] = fact * nu; C[2][1] = fact * nu; C[2][2] = fact * (1 - nu);
    C[3][3] = fact * (1 - 2 * nu) / 2;
    C[4][4] = fact * (1 - 2 * nu) / 2;
    C[5][5] = fact * (1 - 2 * nu) / 2;
    const double gp[2] = {-1 / sqrt(3.0), 1 / sqrt(3.0)};
    double acc = 0.0;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++) {
                const double xi = gp[i], eta = gp[j], zeta = gp[k];
                const double weight = 1.0 * 1.0 * 1.0;
                double dN[8][3] = {
                    {-(1 - eta) * (1 - zeta), -(1 - xi) * (1 - zeta), -(1 - xi) * (1 - eta)},
                    {(1 - eta) * (1 - zeta), -(1 + xi) * (1 - zeta), -(1 + xi) * (1 - eta)},
                    {(1 + eta) * (1 - zeta), (1 + xi) * (1 - zeta), -(1 + xi) * (1 + eta)},
                    {-(1 + eta) * (1 - zeta), (1 - xi) * (1 - zeta), -(1 - xi) * (1 + eta)},
                    {-(1 - eta) * (1 + zeta), -(1 - xi) * (1 + zeta), (1 - xi) * (1 - eta)},
                    {(1 - eta) * (1 + zeta), -(1 + xi) * (1 + zeta), (1 + xi) * (1 - eta)},
                    {(1 + eta) * (1 + zeta), (1 + xi) * (1 + zeta), (1 + xi) * (1 + eta)},
                    {-(1 + eta) * (1 + zeta), (1 - xi) * (1 + zeta), (1 - xi) * (1 + eta)}};
                for (int a = 0; a < 8; a++)
                    for (int q = 0; q < 3; q++) dN[a][q] *= 0.125;
                double B[6][24];
                for (int a = 0; a < 6; a++)
                    for (int b = 0; b < 24; b++) B[a][b] = 0.0;
                for (int a = 0; a < 8; a++) {
                    const int col = a * 3;
                    B[0][col] = dN[a][0];
                    B[1][col + 1] = dN[a][1];
                    B[2][col + 2] = dN[a][2];
                    B[3][col] = dN[a][1];
                    B[3][col + 1] = dN[a][0];
                    B[4][col + 1] = dN[a][2];
                    B[4][col + 2] = dN[a][1];
                    B[5][col] = dN[a][2];
                    B[5][col + 2] = dN[a][0];
                }
                for (int p = 0; p < 6; p++) {
                    double cb = 0.0;
                    for (int q = 0; q < 6; q++) cb += C[p][q] * B[q][n];
                    acc += B[p][m] * cb * 1.0 * weight;
                }
            }
    Ke[t] = acc;
}

// applyAEbe3D / ebePCG general path, step 1: y[a*es + i] = E_e * sum_j Ke[i][j] p[edof_e[j]]
// for element e = elist[a] (explicit list) or e = a (all elements, inactive -> 0).
__global__ void k_elem_products(const double *__restrict__ Ke, int es, const int32_t *__restrict__ edofs,
                                const double *__restrict__ evals, const int32_t *__restrict__ elist, int count,
                                double thresh, const double *__restrict__ p, double *__restrict__ y,
                                const CGState *st) {
    if (st && st->done) return;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)count * es) return;
    const int a = (int)(t / es), i = (int)(t % es);
    const int e = elist ? elist[a] : a;
    const double E = evals[e];
    if (!elist && !(E > thresh)) {
        y[t] = 0.0;
        return;
    }
    const int32_t *ed = edofs + (long long)e * es;
    double sum = 0.0;
    for (int j = 0; j < es; j++) sum += Ke[i * es + j] * p[ed[j]];
    y[t] = E * sum;
}

// step 2: out[d] = sum of its element products in list order, starting from 0.
__global__ void k_csr_gather(const int64_t *__restrict__ rowptr, const int64_t *__restrict__ cols,
                             const double *__restrict__ y, int ndof, double *__restrict__ out,
                             const uint8_t *__restrict__ fixed, const CGState *st) {
    if (st && st->done) return;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= ndof) return;
    double s = 0.0;
    for (int64_t k = rowptr[d]; k < rowptr[d + 1]; k++) s = s + y[cols[k]];
    out[d] = (fixed && fixed[d]) ? 0.0 : s;
}

// ebePCG step 1 (:540-550): stiffness per element with Math.pow.
__global__ void k_ebe_evals(const double *__restrict__ dens, int nel, double Emin, double E0, double penal,
                            double *__restrict__ E) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nel) return;
    E[e] = Emin + pow(dens[e], penal) * (E0 - Emin);
}

// ebePCG step 2 (:552-566): diagonal contributions of active elements.
__global__ void k_diag_general(const double *__restrict__ Ke, int es, const int32_t *__restrict__ edofs,
                               const double *__restrict__ evals, int nel, double thresh,
                               double *__restrict__ ydiag) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nel * es) return;
    const int e = (int)(t / es), i = (int)(t % es);
    const double E = evals[e];
    ydiag[t] = E > thresh ? E * Ke[i * es + i] : 0.0;
}

__global__ void k_invdiag_general(const double *__restrict__ diag, const uint8_t *__restrict__ fixed, int n,
                                  double *__restrict__ invD) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = diag[i];
    invD[i] = (!fixed[i] && d > 1e-30) ? 1.0 / d : 0.0;
}

// denseMatVecRaw (assembly/index.ts:450-464): one thread per row, sequential sum.
__global__ void k_dense_matvec_seq(const double *__restrict__ K, int n, const double *__restrict__ p,
                                   double *__restrict__ Ap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *Kr = K + (long long)i * n;
    double s = 0.0;
    for (int j = 0; j < n; j++) s += Kr[j] * p[j];
    Ap[i] = s;
}

// prepareFilter Hs (:3006-3050): float accumulation in the triplet order
// (neighbour x outer, y, z inner).  One thread per element, reference element order.
__global__ void k_filter_hs(Grid g, double rmin, float *__restrict__ Hs) {
    const long long e1 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e1 >= g.nel) return;
    const int i = (int)(e1 % g.nelx);
    const long long r = e1 / g.nelx;
    const int j = (int)(r % g.nely);
    const int m = (int)(r / g.nely);
    const int R = (int)floor(rmin);
    float acc = 0.0f;
    for (int k = max(i - R, 0); k <= min(i + R, g.nelx - 1); k++)
        for (int l = max(j - R, 0); l <= min(j + R, g.nely - 1); l++)
            for (int n = max(m - R, 0); n <= min(m + R, g.nelz - 1); n++) {
                const double dist = sqrt((double)((i - k) * (i - k) + (j - l) * (j - l) + (m - n) * (m - n)));
                if (dist <= rmin) acc = (float)((double)acc + js_max(0.0, rmin - dist));
            }
    Hs[e1] = acc;
}

// filterSensitivities (:3052-3064): dcn_i = sum_j H_ij x_j dc_j (float accumulation in
// triplet order) / (Hs_i * max(1e-3, x_i)).
__global__ void k_filter_sens(Grid g, double rmin, const float *__restrict__ Hs, const float *__restrict__ x,
                              const float *__restrict__ dc, float *__restrict__ dcn) {
    const long long e1 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e1 >= g.nel) return;
    const int i = (int)(e1 % g.nelx);
    const long long r = e1 / g.nelx;
    const int j = (int)(r % g.nely);
    const int m = (int)(r / g.nely);
    const int R = (int)floor(rmin);
    const long long sy = g.nelx, sz = (long long)g.nelx * g.nely;
    float acc = 0.0f;
    for (int k = max(i - R, 0); k <= min(i + R, g.nelx - 1); k++)
        for (int l = max(j - R, 0); l <= min(j + R, g.nely - 1); l++)
            for (int n = max(m - R, 0); n <= min(m + R, g.nelz - 1); n++) {
                const double dist = sqrt((double)((i - k) * (i - k) + (j - l) * (j - l) + (m - n) * (m - n)));
                if (dist <= rmin) {
                    const long long e2 = k + l * sy + n * sz;
                    const double s = js_max(0.0, rmin - dist);
                    acc = (float)((double)acc + s * (double)__ldg(&x[e2]) * (double)__ldg(&dc[e2]));
                }
            }
    dcn[e1] = (float)((double)acc / ((double)Hs[e1] * js_max(1e-3, (double)x[e1])));
}

// applyDensityFilter (assembly/index.ts:224-273): +-ceil(r) box, dist^2 <= r^2, z outer.
__global__ void k_density_filter(Grid g, double radius, const double *__restrict__ in, double *__restrict__ out) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= g.nel) return;
    const int ex = (int)(e % g.nelx);
    const long long r = e / g.nelx;
    const int ey = (int)(r % g.nely);
    const int ez = (int)(r / g.nely);
    const int R = (int)ceil(radius);
    const double r2 = radius * radius;
    double sum = 0.0, sw = 0.0;
    for (int kz = max(0, ez - R); kz <= min(g.nelz - 1, ez + R); kz++)
        for (int ky = max(0, ey - R); ky <= min(g.nely - 1, ey + R); ky++)
            for (int kx = max(0, ex - R); kx <= min(g.nelx - 1, ex + R); kx++) {
                const double dx = ex - kx, dy = ey - ky, dz = ez - kz;
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 <= r2) {
                    const double w = radius - sqrt(d2);
                    sum += w * __ldg(&in[kx + (long long)ky * g.nelx + (long long)kz * g.nelx * g.nely]);
                    sw += w;
                }
            }
    out[e] = sum / sw;
}

// ---- OC bisection (:3066-3101) --------------------------------------------------------
__device__ __forceinline__ float oc_xnew(float xf, float dcf, const uint8_t *pres, const uint8_t *voidm,
                                         long long i, double lmid) {
    if (pres && pres[i]) return 1.0f;
    if (voidm && voidm[i]) return 0.0f;
    const double x = (double)xf;
    const double Be = -(double)dcf / lmid;
    return (float)js_max(0.0, js_max(x - 0.2, js_min(1.0, js_min(x + 0.2, x * sqrt(Be)))));
}

__global__ void k_oc_init(OCState *s) {
    if (threadIdx.x || blockIdx.x) return;
    s->l1 = 0.0;
    s->l2 = 1e9;
    s->lmid = 0.0;
    s->last_lmid = 0.0;
    s->sum = 0.0;
    s->nb = 0;
    s->counter = 0u;
    s->done = !((s->l2 - s->l1) / (s->l2 + s->l1) > 1e-3);
}

// One bisection step: lmid = (l1 + l2)/2, sum xnew(lmid), move the bracket.
__global__ void k_oc_step(const float *__restrict__ x, const float *__restrict__ dc,
                          const uint8_t *__restrict__ pres, const uint8_t *__restrict__ voidm, long long n,
                          double volfrac, OCState *s, double *partials) {
    if (s->done) return;
    const double lmid = 0.5 * (s->l2 + s->l1);
    double v[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[0] += (double)oc_xnew(x[i], dc[i], pres, voidm, i, lmid);
    __shared__ double sh[32];
    double tot[1];
    if (grid_sum<1>(v, partials, &s->counter, sh, tot) && threadIdx.x == 0) {
        s->sum = tot[0];
        s->last_lmid = lmid;
        if (tot[0] > volfrac * (double)n) s->l1 = lmid;
        else s->l2 = lmid;
        s->nb += 1;
        if (!((s->l2 - s->l1) / (s->l2 + s->l1) > 1e-3)) s->done = 1;
    }
}

// xnew at the last evaluated lmid; change = max |xnew - xold| (exact, order-free max).
__global__ void k_oc_write(const float *__restrict__ x, const float *__restrict__ dc,
                           const uint8_t *__restrict__ pres, const uint8_t *__restrict__ voidm, long long n,
                           const OCState *s, const float *__restrict__ xold, float *__restrict__ xnew,
                           unsigned long long *change_bits) {
    const double lmid = s->last_lmid;
    double mx = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float v = oc_xnew(x[i], dc[i], pres, voidm, i, lmid);
        xnew[i] = v;
        if (xold) mx = js_max(mx, fabs((double)v - (double)xold[i]));
    }
    if (change_bits) {
        // non-negative doubles order like their bit patterns
        unsigned long long b = (unsigned long long)__double_as_longlong(mx);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long ob = __shfl_xor_sync(0xffffffffu, b, o);
            b = ob > b ? ob : b;
        }
        if ((threadIdx.x & 31) == 0) atomicMax(change_bits, b);
    }
}

}  // namespace tpo
