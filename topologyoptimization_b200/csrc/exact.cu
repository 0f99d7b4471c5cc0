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

// Steps 1 and 2 in one launch for the structured element list (no active list): DOF d
// forms each of its element products (e, i) as k_elem_products does and adds them in CSR
// order as k_csr_gather does, so the result is theirs bit for bit.  Every product belongs
// to exactly one DOF, so none is computed twice.
__global__ void k_csr_apply(const double *__restrict__ Ke, int es, const int32_t *__restrict__ edofs,
                            const double *__restrict__ evals, double thresh, const double *__restrict__ p,
                            const int64_t *__restrict__ rowptr, const int64_t *__restrict__ cols, int ndof,
                            double *__restrict__ out, const uint8_t *__restrict__ fixed, const CGState *st) {
    if (st && st->done) return;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= ndof) return;
    double s = 0.0;
    for (int64_t k = rowptr[d]; k < rowptr[d + 1]; k++) {
        const long long t = cols[k];
        const int e = (int)(t / es), i = (int)(t % es);
        const double E = evals[e];
        double y = 0.0;
        if (E > thresh) {
            const int32_t *ed = edofs + (long long)e * es;
            double sum = 0.0;
            for (int j = 0; j < es; j++) sum += Ke[i * es + j] * p[ed[j]];
            y = E * sum;
        }
        s = s + y;
    }
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

// ---- shared-memory tiled filters ---------------------------------------------------------
// A CTA owns an 8x8x8 block of elements and stages the block with its halo of R elements
// per side into shared memory once; the stencil weights, which depend only on the offset,
// come from a table built once per CTA.  Every element then sums its neighbours from
// shared memory in the same order and with the same roundings as the one-thread-per-element
// kernels above (bit-identical results).  Tiles of FT^3 elements, 512 threads.
constexpr int kFT = 8;

// The stencil as a compact list in the loop order of the per-element kernel: the offsets
// inside the radius (packed 8-bit dx, dy, dz), their shared-memory distance from the centre
// element and their weights.  At most (2R+1)^3 entries.
struct FilterTap {
    int packed;  // (dx + 128) | (dy + 128) << 8 | (dz + 128) << 16
    int soff;    // shared-memory offset from the centre element
};
__device__ __forceinline__ int tap_d(int packed, int k) { return ((packed >> (8 * k)) & 255) - 128; }

// filterSensitivities with the +-floor(rmin) box of prepareFilter; R = floor(rmin) <= 4.
// Neighbour order: x outer, y, z inner.
__global__ void __launch_bounds__(512) k_filter_sens_tiled(Grid g, double rmin, const float *__restrict__ Hs,
                                                           const float *__restrict__ x, const float *__restrict__ dc,
                                                           float *__restrict__ dcn) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int R = (int)floor(rmin);
    const int W = 2 * R + 1, T = kFT + 2 * R, W3 = W * W * W;
    double *wt = reinterpret_cast<double *>(smem_raw);  // W^3 tap weights
    FilterTap *taps = reinterpret_cast<FilterTap *>(wt + W3);
    float *sx = reinterpret_cast<float *>(taps + W3);
    float *sd = sx + T * T * T;
    __shared__ int ntaps;
    const int ox = blockIdx.x * kFT, oy = blockIdx.y * kFT, oz = blockIdx.z * kFT;
    if (threadIdx.x < 32) {  // taps in the per-element loop order, compacted by warp 0
        int n = 0;
        for (int c0 = 0; c0 < W3; c0 += 32) {
            const int t = c0 + (int)threadIdx.x;
            const int dk = t / (W * W) - R, dl = (t / W) % W - R, dn = t % W - R;
            const double dist = sqrt((double)(dk * dk + dl * dl + dn * dn));
            const bool in = t < W3 && dist <= rmin;
            const unsigned ball = __ballot_sync(0xffffffffu, in);
            if (in) {
                const int q = n + __popc(ball & ((1u << threadIdx.x) - 1u));
                wt[q] = js_max(0.0, rmin - dist);
                taps[q].packed = (dk + 128) | ((dl + 128) << 8) | ((dn + 128) << 16);
                taps[q].soff = (dn * T + dl) * T + dk;
            }
            n += __popc(ball);
        }
        if (threadIdx.x == 0) ntaps = n;
    }
    for (int t = threadIdx.x; t < T * T * T; t += blockDim.x) {
        const int lx = t % T, ly = (t / T) % T, lz = t / (T * T);
        const int gx = ox - R + lx, gy = oy - R + ly, gz = oz - R + lz;
        if (gx >= 0 && gx < g.nelx && gy >= 0 && gy < g.nely && gz >= 0 && gz < g.nelz) {
            const long long e2 = gx + (long long)gy * g.nelx + (long long)gz * g.nelx * g.nely;
            sx[t] = x[e2];
            sd[t] = dc[e2];
        }
    }
    __syncthreads();
    const int tx = threadIdx.x % kFT, ty = (threadIdx.x / kFT) % kFT, tz = threadIdx.x / (kFT * kFT);
    const int i = ox + tx, j = oy + ty, m = oz + tz;
    if (i >= g.nelx || j >= g.nely || m >= g.nelz) return;
    const int c = ((tz + R) * T + (ty + R)) * T + (tx + R);
    const bool inner = i >= R && i + R < g.nelx && j >= R && j + R < g.nely && m >= R && m + R < g.nelz;
    float acc = 0.0f;
    for (int q = 0; q < ntaps; q++) {
        const FilterTap tp = taps[q];
        if (!inner) {
            const int k = i + tap_d(tp.packed, 0), l = j + tap_d(tp.packed, 1), n = m + tap_d(tp.packed, 2);
            if (k < 0 || k >= g.nelx || l < 0 || l >= g.nely || n < 0 || n >= g.nelz) continue;
        }
        acc = (float)((double)acc + wt[q] * (double)sx[c + tp.soff] * (double)sd[c + tp.soff]);
    }
    const long long e1 = i + (long long)j * g.nelx + (long long)m * g.nelx * g.nely;
    dcn[e1] = (float)((double)acc / ((double)Hs[e1] * js_max(1e-3, (double)sx[c])));
}

// applyDensityFilter (assembly/index.ts:224-273) with its +-ceil(r) box and dist^2 <= r^2,
// neighbour order z outer, y, x inner; R = ceil(r) <= 4.  mode 0: out = sum w in / sum w
// (the filter); mode 1: out = in / sum w (the first half of the transpose); mode 2: out =
// sum w in (the second half).
__global__ void __launch_bounds__(512) k_density_tiled(Grid g, double radius, int mode, const double *__restrict__ in,
                                                       double *__restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int R = (int)ceil(radius);
    const int W = 2 * R + 1, T = kFT + 2 * R, W3 = W * W * W;
    double *wt = reinterpret_cast<double *>(smem_raw);
    FilterTap *taps = reinterpret_cast<FilterTap *>(wt + W3);
    double *sv = reinterpret_cast<double *>(taps + W3 + (W3 & 1));  // 8-byte aligned after the int pairs
    __shared__ int ntaps;
    const int ox = blockIdx.x * kFT, oy = blockIdx.y * kFT, oz = blockIdx.z * kFT;
    const double r2 = radius * radius;
    if (threadIdx.x < 32) {  // taps in the per-element loop order, compacted by warp 0
        int n = 0;
        for (int c0 = 0; c0 < W3; c0 += 32) {
            const int t = c0 + (int)threadIdx.x;
            const int dz = t / (W * W) - R, dy = (t / W) % W - R, dx = t % W - R;
            // the per-element kernel's d = (ex - kx, ey - ky, ez - kz) = -offset
            const double fx = -dx, fy = -dy, fz = -dz;
            const double d2 = fx * fx + fy * fy + fz * fz;
            const bool in = t < W3 && d2 <= r2;
            const unsigned ball = __ballot_sync(0xffffffffu, in);
            if (in) {
                const int q = n + __popc(ball & ((1u << threadIdx.x) - 1u));
                wt[q] = radius - sqrt(d2);
                taps[q].packed = (dx + 128) | ((dy + 128) << 8) | ((dz + 128) << 16);
                taps[q].soff = (dz * T + dy) * T + dx;
            }
            n += __popc(ball);
        }
        if (threadIdx.x == 0) ntaps = n;
    }
    if (mode != 1) {
        for (int t = threadIdx.x; t < T * T * T; t += blockDim.x) {
            const int lx = t % T, ly = (t / T) % T, lz = t / (T * T);
            const int gx = ox - R + lx, gy = oy - R + ly, gz = oz - R + lz;
            if (gx >= 0 && gx < g.nelx && gy >= 0 && gy < g.nely && gz >= 0 && gz < g.nelz)
                sv[t] = in[gx + (long long)gy * g.nelx + (long long)gz * g.nelx * g.nely];
        }
    }
    __syncthreads();
    const int tx = threadIdx.x % kFT, ty = (threadIdx.x / kFT) % kFT, tz = threadIdx.x / (kFT * kFT);
    const int ex = ox + tx, ey = oy + ty, ez = oz + tz;
    if (ex >= g.nelx || ey >= g.nely || ez >= g.nelz) return;
    const int c = ((tz + R) * T + (ty + R)) * T + (tx + R);
    const bool inner = ex >= R && ex + R < g.nelx && ey >= R && ey + R < g.nely && ez >= R && ez + R < g.nelz;
    double sum = 0.0, sw = 0.0;
    for (int q = 0; q < ntaps; q++) {
        const FilterTap tp = taps[q];
        if (!inner) {
            const int kx = ex + tap_d(tp.packed, 0), ky = ey + tap_d(tp.packed, 1), kz = ez + tap_d(tp.packed, 2);
            if (kx < 0 || kx >= g.nelx || ky < 0 || ky >= g.nely || kz < 0 || kz >= g.nelz) continue;
        }
        const double w = wt[q];
        if (mode != 1) sum += w * sv[c + tp.soff];
        sw += w;
    }
    const long long e = ex + (long long)ey * g.nelx + (long long)ez * g.nelx * g.nely;
    out[e] = mode == 0 ? sum / sw : (mode == 1 ? in[e] / sw : sum);
}

// ---- OC bisection (:3066-3101) --------------------------------------------------------
__device__ __forceinline__ float oc_xnew(float xf, float dcf, const uint8_t *pres, const uint8_t *voidm,
                                         long long i, double lmid, double move) {
    if (pres && pres[i]) return 1.0f;
    if (voidm && voidm[i]) return 0.0f;
    const double x = (double)xf;
    const double Be = -(double)dcf / lmid;
    return (float)js_max(0.0, js_max(x - move, js_min(1.0, js_min(x + move, x * sqrt(Be)))));
}

// ---- exact volume sum of the bisection ------------------------------------------------
// Every float in [0, 1] is an integer multiple of 2^-149, so a sum of up to 2^31 of them
// is an integer below 2^180 in those units: three 64-bit limbs hold it exactly.  Integer
// addition is associative, so the total is the same for every grid shape and block order,
// and it is rounded to double once, to nearest-even, before the reference's comparison
// with volfrac * nel.  A NaN (a positive sensitivity under the square root) makes the sum
// NaN, as in the reference.
struct Exact192 {
    unsigned long long w0, w1, w2;
    unsigned int nan;
};

__device__ __forceinline__ void x192_add(Exact192 &a, const Exact192 &b) {
    const unsigned long long s0 = a.w0 + b.w0;
    const unsigned long long c0 = s0 < a.w0;
    unsigned long long s1 = a.w1 + b.w1;
    unsigned long long c1 = s1 < a.w1;
    s1 += c0;
    c1 += s1 < c0;
    a.w0 = s0;
    a.w1 = s1;
    a.w2 = a.w2 + b.w2 + c1;
    a.nan |= b.nan;
}

// a += v for a float v in [0, 1] (or NaN)
__device__ __forceinline__ void x192_add_float(Exact192 &a, float v) {
    if (v != v) {
        a.nan = 1u;
        return;
    }
    const unsigned bits = __float_as_uint(v) & 0x7fffffffu;  // xnew >= +0; a -0 counts as 0
    const unsigned e = bits >> 23;
    const unsigned long long m = e ? (unsigned long long)((bits & 0x7fffffu) | 0x800000u)
                                   : (unsigned long long)(bits & 0x7fffffu);
    const int sh = e ? (int)e - 1 : 0;  // v = m 2^(sh - 149); sh <= 126 for v <= 1
    const int li = sh >> 6, off = sh & 63;
    Exact192 t{0ULL, 0ULL, 0ULL, 0u};
    const unsigned long long lo = m << off, hi = off > 40 ? m >> (64 - off) : 0ULL;
    if (li == 0) {
        t.w0 = lo;
        t.w1 = hi;
    } else {
        t.w1 = lo;
        t.w2 = hi;
    }
    x192_add(a, t);
}

__device__ __forceinline__ Exact192 x192_shfl_down(const Exact192 &a, int o) {
    Exact192 r;
    r.w0 = __shfl_down_sync(0xffffffffu, a.w0, o);
    r.w1 = __shfl_down_sync(0xffffffffu, a.w1, o);
    r.w2 = __shfl_down_sync(0xffffffffu, a.w2, o);
    r.nan = __shfl_down_sync(0xffffffffu, a.nan, o);
    return r;
}

// 64 bits of W starting at bit s (0 <= s < 192)
__device__ __forceinline__ unsigned long long x192_bits(const Exact192 &a, int s) {
    const unsigned long long w[4] = {a.w0, a.w1, a.w2, 0ULL};
    const int li = s >> 6, off = s & 63;
    return off ? (w[li] >> off) | (w[li + 1] << (64 - off)) : w[li];
}

// W 2^-149 rounded to the nearest double (ties to even)
__device__ double x192_to_double(const Exact192 &a) {
    if (a.nan) return __longlong_as_double(0x7ff8000000000000LL);
    int p = -1;  // highest set bit
    if (a.w2) p = 128 + 63 - __clzll((long long)a.w2);
    else if (a.w1) p = 64 + 63 - __clzll((long long)a.w1);
    else if (a.w0) p = 63 - __clzll((long long)a.w0);
    if (p < 0) return 0.0;
    if (p < 53) return ldexp((double)a.w0, -149);  // exact: W < 2^53
    const int sh = p - 52;
    unsigned long long mant = x192_bits(a, sh) & ((1ULL << 53) - 1ULL);
    const bool round = (x192_bits(a, sh - 1) & 1ULL) != 0;
    bool sticky = false;
    const int below = sh - 1;  // bits [0, below) decide the tie
    {
        const unsigned long long w[3] = {a.w0, a.w1, a.w2};
        for (int li = 0; li < 3 && li * 64 < below; li++) {
            const int nb = below - li * 64;
            const unsigned long long m = nb >= 64 ? ~0ULL : ((1ULL << nb) - 1ULL);
            if (w[li] & m) sticky = true;
        }
    }
    if (round && (sticky || (mant & 1ULL))) mant += 1ULL;  // 2^53 stays exact
    return ldexp((double)mant, sh - 149);
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

// One bisection step: lmid = (l1 + l2)/2, sum xnew(lmid) exactly, move the bracket
// (OC, js/optimizer-worker-3d.js:3066-3101).  partials holds 4 words per block.
__global__ void k_oc_step(const float *__restrict__ x, const float *__restrict__ dc,
                          const uint8_t *__restrict__ pres, const uint8_t *__restrict__ voidm, long long n,
                          double volfrac, double move, OCState *s, double *partials) {
    if (s->done) return;
    const double lmid = 0.5 * (s->l2 + s->l1);
    Exact192 acc{0ULL, 0ULL, 0ULL, 0u};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x192_add_float(acc, oc_xnew(x[i], dc[i], pres, voidm, i, lmid, move));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const Exact192 b = x192_shfl_down(acc, o);
        x192_add(acc, b);
    }
    __shared__ Exact192 sh[32];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = acc;
    __syncthreads();
    unsigned long long *pw = reinterpret_cast<unsigned long long *>(partials);
    if (threadIdx.x == 0) {
        Exact192 b{0ULL, 0ULL, 0ULL, 0u};
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) x192_add(b, sh[w]);
        pw[4 * blockIdx.x + 0] = b.w0;
        pw[4 * blockIdx.x + 1] = b.w1;
        pw[4 * blockIdx.x + 2] = b.w2;
        pw[4 * blockIdx.x + 3] = b.nan;
        __threadfence();
        const unsigned int t = atomicAdd(&s->counter, 1u);
        s_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    Exact192 tot{0ULL, 0ULL, 0ULL, 0u};
    for (unsigned b = 0; b < gridDim.x; b++) {
        const Exact192 pb{__ldcg(&pw[4 * b + 0]), __ldcg(&pw[4 * b + 1]), __ldcg(&pw[4 * b + 2]),
                          (unsigned int)__ldcg(&pw[4 * b + 3])};
        x192_add(tot, pb);
    }
    s->counter = 0u;
    const double sum = x192_to_double(tot);
    s->sum = sum;
    s->last_lmid = lmid;
    if (sum > volfrac * (double)n) s->l1 = lmid;
    else s->l2 = lmid;
    s->nb += 1;
    if (!((s->l2 - s->l1) / (s->l2 + s->l1) > 1e-3)) s->done = 1;
}

// xnew at the last evaluated lmid; change = max |xnew - xold| (exact, order-free max).
__global__ void k_oc_write(const float *__restrict__ x, const float *__restrict__ dc,
                           const uint8_t *__restrict__ pres, const uint8_t *__restrict__ voidm, long long n,
                           double move, const OCState *s, const float *__restrict__ xold, float *__restrict__ xnew,
                           unsigned long long *change_bits) {
    const double lmid = s->last_lmid;
    double mx = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float v = oc_xnew(x[i], dc[i], pres, voidm, i, lmid, move);
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

// _assembleGalerkinFromElements (js/optimizer-worker-3d.js:628-662) as a gather: one
// thread per coarse entry (R, C), no atomics.  The reference scatters, for every active
// fine element in ascending element order, for i, for j >= i, for the prolongation
// pairs (pi, pj): K[cr][cc] += w_i E Ke_ij w_j and, for i != j, K[cc][cr] += the same
// value.  The thread walks the fine elements whose nodes interpolate from both coarse
// nodes in that element order and adds the terms that land on (R, C) in that (i, j, pi,
// pj) order, so the sum is the reference's, bit for bit, and the same on every run.
// The weights are powers of two, so every term is exactly E Ke_ij w w'.
__device__ __forceinline__ void fine_node_range(int c, int nC, int nF, int &lo, int &hi) {
    lo = max(0, 2 * c - 1);
    hi = (c == nC - 1) ? nF - 1 : min(nF - 1, 2 * c + 1);
}
// Position of coarse axis index c in a fine index's prolongation pair: 0 (c0) or 1 (c1).
__device__ __forceinline__ int pair_slot(int f, int c, int nC) { return min(f >> 1, nC - 1) == c ? 0 : 1; }
// Number of positive-weight partners of fine index f along one axis (1, or 2 when t > 0).
__device__ __forceinline__ int pair_count(int f, int nC) {
    const int c0 = min(f >> 1, nC - 1), c1 = min(c0 + 1, nC - 1);
    return (c0 != c1 && (f & 1)) ? 2 : 1;
}

__global__ void k_galerkin_gather(const __grid_constant__ KeParam<double> ke, Grid gf, Grid gc,
                                  const double *__restrict__ EactF, double *__restrict__ Kc) {
    const long long n = gc.ndof;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n * n) return;
    const long long R = t / n, C = t % n;
    const int dR = (int)(R % 3), dC = (int)(C % 3);
    int rx, ry, rz, cx, cy, cz;
    node_xyz(gc, R / 3, rx, ry, rz);
    node_xyz(gc, C / 3, cx, cy, cz);
    int lo[3], hi[3];
    {
        int a, b, c2, d;
        fine_node_range(rx, gc.nnx, gf.nnx, a, b);
        fine_node_range(cx, gc.nnx, gf.nnx, c2, d);
        lo[0] = max(max(a, c2) - 1, 0);
        hi[0] = min(min(b, d), gf.nelx - 1);
        fine_node_range(ry, gc.nny, gf.nny, a, b);
        fine_node_range(cy, gc.nny, gf.nny, c2, d);
        lo[1] = max(max(a, c2) - 1, 0);
        hi[1] = min(min(b, d), gf.nely - 1);
        fine_node_range(rz, gc.nnz, gf.nnz, a, b);
        fine_node_range(cz, gc.nnz, gf.nnz, c2, d);
        lo[2] = max(max(a, c2) - 1, 0);
        hi[2] = min(min(b, d), gf.nelz - 1);
    }
    double sum = 0.0;
    for (int ez = lo[2]; ez <= hi[2]; ez++)
        for (int ey = lo[1]; ey <= hi[1]; ey++)
            for (int ex = lo[0]; ex <= hi[0]; ex++) {
                const double E = EactF[((long long)ex * gf.nely + ey) * gf.nelz + ez];
                if (E == 0.0) continue;
                double wR[8], wC[8];
                int sR[8], sC[8];  // list positions of the coarse nodes in each node's prolongation
#pragma unroll
                for (int b = 0; b < 8; b++) {
                    const int fx = ex + (b == 1 || b == 2 || b == 5 || b == 6);
                    const int fy = ey + (b == 2 || b == 3 || b == 6 || b == 7);
                    const int fz = ez + (b >= 4);
                    wR[b] = w1d(fx, rx, gc.nnx) * w1d(fy, ry, gc.nny) * w1d(fz, rz, gc.nnz);
                    wC[b] = w1d(fx, cx, gc.nnx) * w1d(fy, cy, gc.nny) * w1d(fz, cz, gc.nnz);
                    // the list runs dz, dy, dx (dx fastest) over the positive weights
                    const int nx = pair_count(fx, gc.nnx), ny = pair_count(fy, gc.nny);
                    sR[b] = (pair_slot(fz, rz, gc.nnz) * ny + pair_slot(fy, ry, gc.nny)) * nx +
                            pair_slot(fx, rx, gc.nnx);
                    sC[b] = (pair_slot(fz, cz, gc.nnz) * ny + pair_slot(fy, cy, gc.nny)) * nx +
                            pair_slot(fx, cx, gc.nnx);
                }
                for (int i = 0; i < 24; i++) {
                    const int bi = i / 3, di = i % 3;
                    const bool iR = di == dR && wR[bi] > 0.0, iC = di == dC && wC[bi] > 0.0;
                    if (!iR && !iC) continue;
                    for (int j = i; j < 24; j++) {
                        const int bj = j / 3, dj = j % 3;
                        const bool dir = iR && dj == dC && wC[bj] > 0.0;
                        const bool tr = iC && i != j && dj == dR && wR[bj] > 0.0;
                        if (!dir && !tr) continue;
                        const double kij = E * ke.v[i * 24 + j];
                        if (kij == 0.0) continue;
                        const double vd = wR[bi] * kij * wC[bj];  // at (pi, pj) = (sR[bi], sC[bj])
                        const double vt = wC[bi] * kij * wR[bj];  // at (pi, pj) = (sC[bi], sR[bj])
                        if (dir && tr) {
                            const bool dfirst = sR[bi] < sC[bi] || (sR[bi] == sC[bi] && sC[bj] <= sR[bj]);
                            if (dfirst) {
                                sum += vd;
                                sum += vt;
                            } else {
                                sum += vt;
                                sum += vd;
                            }
                        } else {
                            sum += dir ? vd : vt;
                        }
                    }
                }
            }
    Kc[t] = sum;
}

// GPUCompute.computeElementEnergies (js/gpu-compute.js:187-303): the reference's WGSL
// kernel, one invocation per element, energy = sum_i sum_j u_i KE_ij u_j in f32 in that
// order, DOF indices < 0 skipped.  Unfused f32 operations (this file is built without
// FMA contraction).
__global__ void k_energy_wgsl(const float *__restrict__ U, const float *__restrict__ KE,
                              const int32_t *__restrict__ edofs, int nel, int es, float *__restrict__ out) {
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= nel) return;
    const long long off = (long long)el * es;
    float energy = 0.0f;
    for (int i = 0; i < es; i++) {
        const int di = edofs[off + i];
        if (di < 0) continue;
        const float ui = U[di];
        for (int j = 0; j < es; j++) {
            const int dj = edofs[off + j];
            if (dj < 0) continue;
            energy = energy + ui * KE[i * es + j] * U[dj];
        }
    }
    out[el] = energy;
}

// ---- the 2D worker's hot path (js/optimizer-worker.js, TopologyOptimizerWorker) ------------
// _precomputeStiffness (:270-285): E = Emin + Math.pow(x, penal) (E0 - Emin) from the float
// (projected) densities, two roundings.
__global__ void k_evals_pow_f32(const float *__restrict__ x, int nel, double Emin, double E0, double penal,
                                double *__restrict__ E) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nel) return;
    E[e] = Emin + pow((double)x[e], penal) * (E0 - Emin);
}

// _computeElementEnergyFlat (:335-345; js/optimizer-worker-3d.js:1561-1571): energy = sum_i
// sum_j u_i KE_ij u_j in FP64 in that order over the element's DOFs, stored as float.
__global__ void k_energy_general(const double *__restrict__ Ke, int es, const int32_t *__restrict__ edofs,
                                 const double *__restrict__ U, int nel, float *__restrict__ energy) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nel) return;
    const int32_t *ed = edofs + (long long)e * es;
    double en = 0.0;
    for (int i = 0; i < es; i++) {
        const double ui = U[ed[i]];
        for (int j = 0; j < es; j++) en += ui * Ke[i * es + j] * U[ed[j]];
    }
    energy[e] = (float)en;
}

// 2D prepareFilter (:1391-1429): element e = i*nely + j (column-major); neighbours k (x)
// outer, l (y) inner within +-floor(rmin), weight max(0, rmin - dist) where dist <= rmin;
// Hs accumulated into a Float32Array.
__global__ void k_filter_hs2d(int nelx, int nely, double rmin, float *__restrict__ Hs) {
    const int e1 = blockIdx.x * blockDim.x + threadIdx.x;
    if (e1 >= nelx * nely) return;
    const int i = e1 / nely, j = e1 % nely;
    const int R = (int)floor(rmin);
    float acc = 0.0f;
    for (int k = max(i - R, 0); k <= min(i + R, nelx - 1); k++)
        for (int l = max(j - R, 0); l <= min(j + R, nely - 1); l++) {
            const double dist = sqrt((double)((i - k) * (i - k) + (j - l) * (j - l)));
            if (dist <= rmin) acc = (float)((double)acc + js_max(0.0, rmin - dist));
        }
    Hs[e1] = acc;
}

// 2D filterSensitivities (:1431-1443): dcn_e = sum H x dc (float accumulation in the
// triplet order) / (Hs_e max(1e-3, x_e)).
__global__ void k_filter_sens2d(int nelx, int nely, double rmin, const float *__restrict__ Hs,
                                const float *__restrict__ x, const float *__restrict__ dc, float *__restrict__ dcn) {
    const int e1 = blockIdx.x * blockDim.x + threadIdx.x;
    if (e1 >= nelx * nely) return;
    const int i = e1 / nely, j = e1 % nely;
    const int R = (int)floor(rmin);
    float acc = 0.0f;
    for (int k = max(i - R, 0); k <= min(i + R, nelx - 1); k++)
        for (int l = max(j - R, 0); l <= min(j + R, nely - 1); l++) {
            const double dist = sqrt((double)((i - k) * (i - k) + (j - l) * (j - l)));
            if (dist <= rmin) {
                const int e2 = k * nely + l;
                acc = (float)((double)acc + js_max(0.0, rmin - dist) * (double)x[e2] * (double)dc[e2]);
            }
        }
    dcn[e1] = (float)((double)acc / ((double)Hs[e1] * js_max(1e-3, (double)x[e1])));
}

}  // namespace tpo
