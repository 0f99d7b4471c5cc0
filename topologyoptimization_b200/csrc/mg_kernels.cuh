// Templated multigrid and vector kernels (FP64 and FP32 instantiations), defined in a
// header so each instantiation lives in the translation unit that launches it.
#pragma once
#include <algorithm>
#include <type_traits>

#include "common.cuh"

namespace tpo {

// Launch shapes of the grid transfers.  Restriction, and prolongation in FP32, run one CTA
// per node line (x, y) of the target grid (blockIdx.x) and one thread per node of the line
// (blockIdx.y chunks of blockDim.x), so a line's coordinates and weights are uniform in
// the CTA and no thread divides by a runtime value.  FP64 prolongation runs one thread per
// fine node over the flat node range, which measured faster for 8-byte values.
inline unsigned transfer_threads(const Grid &g) { return (unsigned)std::min(256, (g.nnz + 31) / 32 * 32); }
inline dim3 restrict_grid(const Grid &gc, unsigned nrhs) {
    const unsigned b = transfer_threads(gc);
    return dim3((unsigned)((long long)gc.nnx * gc.nny), (gc.nnz + b - 1) / b, nrhs);
}
inline dim3 restrict_block(const Grid &gc) { return dim3(transfer_threads(gc), 1, 1); }
template <typename T>
dim3 prolong_grid(const Grid &gf, unsigned nrhs) {
    if (std::is_same_v<T, double>) return dim3((unsigned)((gf.nnodes + 255) / 256), 1, nrhs);
    const unsigned b = transfer_threads(gf);
    return dim3((unsigned)((long long)gf.nnx * gf.nny), (gf.nnz + b - 1) / b, nrhs);
}
template <typename T>
dim3 prolong_block(const Grid &gf) {
    return dim3(std::is_same_v<T, double> ? 256u : transfer_threads(gf), 1, 1);
}

// Restriction bC = P^T res (gather form), one thread per coarse node.  Contributions to
// one coarse DOF are added in the reference's fine-node order (fz, fy, fx ascending);
// weights are powers of two, so the result equals the reference's scatter loop bit for
// bit.  Each fine z-plane's 27 values are loaded unconditionally (indices outside the grid
// clamped to its edge, their terms then skipped), so they are in flight together.
template <typename T>
__global__ void k_restrict(Grid gf, Grid gc, const T *__restrict__ res, const uint8_t *__restrict__ fixedC,
                           T *__restrict__ bC, const CGState *st) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    res += zr * gf.ndof;
    bC += zr * gc.ndof;
    if (st) st += zr;
    if (st && st->done) return;
    const int cz = blockIdx.y * blockDim.x + threadIdx.x;
    if (cz >= gc.nnz) return;
    const int line = blockIdx.x;
    const int cx = line / gc.nny, cy = line - cx * gc.nny;
    // the fine nodes 2c-1, 2c, 2c+1 along each axis with their weights (0 outside the grid)
    T wz[3], wy[3], wx[3];
    int fz[3], fy[3], fx[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const int f = 2 * cz + k - 1;
        const bool in = f >= 0 && f < gf.nnz;
        wz[k] = in ? (T)w1d(f, cz, gc.nnz) : T(0);
        fz[k] = in ? f : 2 * cz;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const int f = 2 * cy + k - 1;
        const bool in = f >= 0 && f < gf.nny;
        wy[k] = in ? (T)w1d(f, cy, gc.nny) : T(0);
        fy[k] = in ? f : 2 * cy;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const int f = 2 * cx + k - 1;
        const bool in = f >= 0 && f < gf.nnx;
        wx[k] = in ? (T)w1d(f, cx, gc.nnx) : T(0);
        fx[k] = in ? f : 2 * cx;
    }
    const long long lw = 3LL * gf.nnz;
    const T *row[3][3];
#pragma unroll
    for (int ix = 0; ix < 3; ix++)
#pragma unroll
        for (int iy = 0; iy < 3; iy++) row[ix][iy] = res + ((long long)fx[ix] * gf.nny + fy[iy]) * lw;
    T s[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int iz = 0; iz < 3; iz++) {
        T v[3][3][3];
#pragma unroll
        for (int iy = 0; iy < 3; iy++)
#pragma unroll
            for (int ix = 0; ix < 3; ix++)
#pragma unroll
                for (int d = 0; d < 3; d++) v[iy][ix][d] = __ldg(row[ix][iy] + 3 * fz[iz] + d);
#pragma unroll
        for (int iy = 0; iy < 3; iy++)
#pragma unroll
            for (int ix = 0; ix < 3; ix++) {
                // products of powers of two: exact, as the reference's weight
                const T w = wx[ix] * wy[iy] * wz[iz];
#pragma unroll
                for (int d = 0; d < 3; d++) s[d] = w != T(0) ? s[d] + w * v[iy][ix][d] : s[d];
            }
    }
    const long long q = ((long long)line * gc.nnz + cz) * 3;
#pragma unroll
    for (int d = 0; d < 3; d++) bC[q + d] = fixedC[q + d] ? T(0) : s[d];
}

// Prolongation x += P xC on free fine DOFs, one thread per fine node, corner order
// 000,100,010,110,001,101,011,111.  Per axis the fine node sits on coarse node c0
// (weight 1), or halfway between c0 and c0 + 1 (weight 1/2 each; w1d of common.cuh).
// Corners of weight 0 are skipped: the sum runs over the remaining corners in the order
// 000,100,...,111, so it rounds exactly as the full 8-term sum with its zero terms.  The
// corner values, x and the mask are loaded unconditionally (a missing corner reads c0
// again), so the loads are in flight together.
template <typename T>
__global__ void k_prolong(Grid gf, Grid gc, const T *__restrict__ xC, const uint8_t *__restrict__ fixedF,
                          T *__restrict__ x, const CGState *st) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    xC += zr * gc.ndof;
    x += zr * gf.ndof;
    if (st) st += zr;
    if (st && st->done) return;
    long long f;
    int fx, fy, fz;
    if constexpr (std::is_same_v<T, double>) {
        f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        if (f >= gf.nnodes) return;
        node_xyz(gf, f, fx, fy, fz);
    } else {
        fz = blockIdx.y * blockDim.x + threadIdx.x;
        if (fz >= gf.nnz) return;
        const int line = blockIdx.x;
        fx = line / gf.nny;
        fy = line - fx * gf.nny;
        f = (long long)line * gf.nnz + fz;
    }
    const int cx0 = min(fx >> 1, gc.nnx - 1), cy0 = min(fy >> 1, gc.nny - 1), cz0 = min(fz >> 1, gc.nnz - 1);
    const bool bx = cx0 + 1 < gc.nnx && (fx & 1);
    const bool by = cy0 + 1 < gc.nny && (fy & 1);
    const bool bz = cz0 + 1 < gc.nnz && (fz & 1);
    const T w = (T)((bx ? 0.5 : 1.0) * (by ? 0.5 : 1.0) * (bz ? 0.5 : 1.0));
    const long long lw = 3LL * gc.nnz;
    const T *c00 = xC + ((long long)cx0 * gc.nny + cy0) * lw + 3 * cz0;
    const long long ox = bx ? (long long)gc.nny * lw : 0, oy = by ? lw : 0;
    const int oz = bz ? 3 : 0;
    const long long q = 3 * f;
    uint8_t fm[3];
    T xq[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        fm[d] = fixedF[q + d];
        xq[d] = x[q + d];
    }
    T c[8][3];
#pragma unroll
    for (int k = 0; k < 8; k++)
#pragma unroll
        for (int d = 0; d < 3; d++)
            c[k][d] = __ldg(c00 + ((k & 1) ? ox : 0) + ((k & 2) ? oy : 0) + ((k & 4) ? oz : 0) + d);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        T val = c[0][d] * w;
#pragma unroll
        for (int k = 1; k < 8; k++) {
            const bool on = (!(k & 1) || bx) && (!(k & 2) || by) && (!(k & 4) || bz);
            val = on ? val + c[k][d] * w : val;
        }
        if (!fm[d]) x[q + d] = xq[d] + val;
    }
}

// Damped Jacobi on a dense level, one warp per row (mgSmooth with mgApplyA dense path).
template <typename T>
__global__ void k_dense_smooth(const double *__restrict__ K, int n, const T *__restrict__ x, const T *__restrict__ b,
                               const T *__restrict__ invD, const uint8_t *__restrict__ fixed, T omega,
                               const double *__restrict__ womega, T *__restrict__ xn, const CGState *st) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    x += zr * n;
    b += zr * n;
    xn += zr * n;
    if (st) st += zr;
    if (st && st->done) return;
    const double w = womega ? *womega : (double)omega;  // womega: damping set on the device per update
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const double *Kr = K + (long long)row * n;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += Kr[j] * (double)x[j];
    s = warp_sum(s);
    if (lane == 0) {
        const T xi = x[row];
        xn[row] = fixed[row] ? xi : (T)((double)xi + w * (double)invD[row] * ((double)b[row] - s));
    }
}
template <typename T>
__global__ void k_dense_residual(const double *__restrict__ K, int n, const T *__restrict__ x, const T *__restrict__ b,
                                 const uint8_t *__restrict__ fixed, T *__restrict__ res, const CGState *st) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    x += zr * n;
    b += zr * n;
    res += zr * n;
    if (st) st += zr;
    if (st && st->done) return;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const double *Kr = K + (long long)row * n;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += Kr[j] * (double)x[j];
    s = warp_sum(s);
    if (lane == 0) res[row] = fixed[row] ? T(0) : (T)((double)b[row] - s);
}

// ---- vectors ------------------------------------------------------------------------
template <typename T>
__global__ void k_zero(T *a, long long n, const CGState *st) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    a += zr * n;
    if (st) st += zr;
    if (st && st->done) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] = T(0);
}
template <typename T>
__global__ void k_copy(const T *__restrict__ a, T *__restrict__ b, long long n, const CGState *st) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    a += zr * n;
    b += zr * n;
    if (st) st += zr;
    if (st && st->done) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = a[i];
}
// First smoothing sweep from x = 0: x = 0 + omega*invD*(b - A*0), so no operator apply.
template <typename T>
__global__ void k_smooth0(const T *__restrict__ b, const T *__restrict__ invD, const uint8_t *__restrict__ fixed,
                          T omega, const double *__restrict__ womega, T *__restrict__ x, long long n,
                          const CGState *st) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    b += zr * n;
    x += zr * n;
    if (st) st += zr;
    if (st && st->done) return;
    const T w = womega ? (T)*womega : omega;
    // 16-byte vectors where every array is aligned for them (a batched right-hand side
    // whose offset is not leaves the scalar loop to do all of it)
    constexpr int V = 16 / sizeof(T);
    using Vec = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    using Fx = typename std::conditional<sizeof(T) == 4, uchar4, uchar2>::type;
    const bool vec_ok = ((reinterpret_cast<unsigned long long>(b) | reinterpret_cast<unsigned long long>(invD) |
                          reinterpret_cast<unsigned long long>(x)) & 15ULL) == 0 &&
                        (reinterpret_cast<unsigned long long>(fixed) & (unsigned long long)(V - 1)) == 0;
    const long long nv = vec_ok ? n / V : 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += stride) {
        const Vec bv = reinterpret_cast<const Vec *>(b)[i];
        const Vec dv = reinterpret_cast<const Vec *>(invD)[i];
        const Fx fv = reinterpret_cast<const Fx *>(fixed)[i];
        const T *bs = reinterpret_cast<const T *>(&bv);
        const T *ds = reinterpret_cast<const T *>(&dv);
        const unsigned char *fs = reinterpret_cast<const unsigned char *>(&fv);
        Vec xv;
        T *xs = reinterpret_cast<T *>(&xv);
#pragma unroll
        for (int j = 0; j < V; j++) xs[j] = fs[j] ? T(0) : T(0) + w * ds[j] * bs[j];
        reinterpret_cast<Vec *>(x)[i] = xv;
    }
    for (long long i = nv * V + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride)
        x[i] = fixed[i] ? T(0) : T(0) + w * invD[i] * b[i];
}

// ---- PCG on T-precision vectors with FP64 scalars (inner solve of the mixed-precision
// defect correction; same recurrences as k_cg_* of kernels.cu) --------------------------
template <typename T>
__global__ void k_cgT_rr(const T *__restrict__ r, long long n, CGState *st, double *partials) {
    double v[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double ri = (double)r[i];
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

template <typename T>
__global__ void k_cgT_pz(const T *__restrict__ r, T *__restrict__ z, const uint8_t *__restrict__ fixed,
                         T *__restrict__ p, long long n, CGState *st, double *partials) {
    if (st->done) return;
    double v[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        T zi = z[i];
        if (fixed[i]) zi = T(0);
        z[i] = zi;
        p[i] = zi;
        v[0] += (double)r[i] * (double)zi;
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

template <typename T>
__global__ void k_cgT_update(T *__restrict__ d, T *__restrict__ r, const T *__restrict__ p, const T *__restrict__ Ap,
                             long long n, CGState *st, double *partials) {
    if (st->done) return;
    const T alpha = (T)st->alpha;
    double v[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        d[i] = d[i] + alpha * p[i];
        const T ri = r[i] - alpha * Ap[i];
        r[i] = ri;
        v[0] += (double)ri * (double)ri;
    }
    __shared__ double sh[32];
    double tot[1];
    if (grid_sum<1>(v, partials, &st->counters[2], sh, tot) && threadIdx.x == 0) {
        st->rr = tot[0];
        cg_decide(st);
    }
}

template <typename T>
__global__ void k_cgT_rz(const T *__restrict__ r, T *__restrict__ z, const uint8_t *__restrict__ fixed, long long n,
                         CGState *st, double *partials) {
    if (st->done) return;
    double v[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        T zi = z[i];
        if (fixed[i]) {
            zi = T(0);
            z[i] = zi;
        }
        v[0] += (double)r[i] * (double)zi;
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

template <typename T>
__global__ void k_cgT_p(T *__restrict__ p, const T *__restrict__ z, long long n, const CGState *st) {
    if (st->done) return;
    const T beta = (T)st->beta;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

// U += d (the FP32 correction accumulated into the FP64 solution).
__global__ void k_add_f32_to_f64(double *__restrict__ U, const float *__restrict__ d, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        U[i] += (double)d[i];
}

// ---- mixed precision with reliable updates ---------------------------------------------
__global__ void k_rel_setup(CGState *st, double tol, int maxIter, double delta) {
    if (threadIdx.x || blockIdx.x) return;
    st->rz = st->rz_new = st->pAp = st->alpha = st->beta = st->rr = st->r0 = 0.0;
    st->tolSq = tol;  // squared against the initial residual by the first EpiDefect
    st->eps = 0.0;
    st->it = st->done = st->iters = st->converged = st->nonfinite = 0;
    st->maxIter = maxIter;
    st->rr32 = 0.0;
    st->maxr2 = 0.0;
    st->delta2 = delta * delta;
    st->do_update = 1;  // the first defect computes the initial residual
    st->n_updates = 0;
    for (int k = 0; k < 8; k++) st->counters[k] = 0u;
}

// x += alpha p; r -= alpha Ap (FP32); ||r||^2 in FP64.  Asks for a reliable update when the
// recursive residual fell by delta since the last one, reached the tolerance, or the
// iteration cap is hit.
template <typename T>
__global__ void k_cgR_update(T *__restrict__ x, T *__restrict__ r, const T *__restrict__ p, const T *__restrict__ Ap,
                             long long n, CGState *st, double *partials) {
    if (st->done) return;
    const T alpha = (T)st->alpha;
    double v[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        x[i] = x[i] + alpha * p[i];
        const T ri = r[i] - alpha * Ap[i];
        r[i] = ri;
        v[0] += (double)ri * (double)ri;
    }
    __shared__ double sh[32];
    double tot[1];
    if (grid_sum<1>(v, partials, &st->counters[2], sh, tot) && threadIdx.x == 0) {
        st->rr32 = tot[0];
        st->it += 1;
        if (!isfinite(tot[0])) {
            st->nonfinite = 1;
            st->done = 1;
            st->iters = st->it;
        } else if (tot[0] < st->delta2 * st->maxr2 || tot[0] < st->tolSq || st->it >= st->maxIter) {
            st->do_update = 1;
        }
    }
}

// U += x (FP64), x = 0, when an update is due.
__global__ void k_rel_merge(double *__restrict__ U, float *__restrict__ x, long long n, const CGState *st) {
    if (st->done || !st->do_update) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        U[i] += (double)x[i];
        x[i] = 0.f;
    }
}

// ---- FP64 PCG with the FP32 multigrid preconditioner ------------------------------------
// r32 = (float) r, the V-cycle's input.
__global__ void k_cgP_init(const double *__restrict__ r, float *__restrict__ r32, long long n) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    r += zr * n;
    r32 += zr * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        r32[i] = (float)r[i];
}

// p = z32 (masked); rz = r.z32; initial convergence test (k_cg_pz of the FP64 solve).
__global__ void k_cgP_pz(const double *__restrict__ r, float *__restrict__ z32, const uint8_t *__restrict__ fixed,
                         double *__restrict__ p, long long n, CGState *st, double *partials) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    r += zr * n;
    z32 += zr * n;
    p += zr * n;
    st += zr;
    if (st->done) return;
    double v[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double zi = fixed[i] ? 0.0 : (double)z32[i];
        z32[i] = (float)zi;
        p[i] = zi;
        v[0] += r[i] * zi;
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

// U += alpha p; r -= alpha Ap (FP64); r32 = (float) r; ||r||^2; convergence decision.
__global__ void k_cgP_update(double *__restrict__ U, double *__restrict__ r, float *__restrict__ r32,
                             const double *__restrict__ p, const double *__restrict__ Ap, long long n, CGState *st,
                             double *partials) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    U += zr * n;
    r += zr * n;
    r32 += zr * n;
    p += zr * n;
    Ap += zr * n;
    st += zr;
    if (st->done) return;
    const double alpha = st->alpha;
    double v[1] = {0.0};
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
    const bool vec = aligned_to(16, U, r, p, Ap) && aligned_to(8, r32);
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
        st_pair(r32, i, Pair<float>{(float)rr.x, (float)rr.y}, vec);
        v[0] += rr.x * rr.x;
        v[0] += rr.y * rr.y;
    }
    for (long long i = 2 * nv + t0; i < n; i += stride) {
        U[i] = U[i] + alpha * p[i];
        const double ri = r[i] - alpha * Ap[i];
        r[i] = ri;
        r32[i] = (float)ri;
        v[0] += ri * ri;
    }
    __shared__ double sh[32];
    double tot[1];
    if (grid_sum<1>(v, partials, &st->counters[2], sh, tot) && threadIdx.x == 0) {
        st->rr = tot[0];
        cg_decide(st);
    }
}

// z32 zeroed on fixed DOFs; rz_new = r.z32 (FP64); beta.
__global__ void k_cgP_rz(const double *__restrict__ r, float *__restrict__ z32, const uint8_t *__restrict__ fixed,
                         long long n, CGState *st, double *partials) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    r += zr * n;
    z32 += zr * n;
    st += zr;
    if (st->done) return;
    double v[1] = {0.0};
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
    const bool vec = aligned_to(16, r) && aligned_to(8, z32);
    const long long nv = n / 2;
    for (long long i = t0; i < nv; i += stride) {  // pairs of DOFs
        const Pair<double> rr = ld_pair(r, i, vec);
        Pair<float> zz = ld_pair(z32, i, vec);
        const uint8_t f0 = fixed[2 * i], f1 = fixed[2 * i + 1];
        if (f0 || f1) {
            if (f0) zz.x = 0.f;
            if (f1) zz.y = 0.f;
            st_pair(z32, i, zz, vec);
        }
        v[0] += rr.x * (double)zz.x;
        v[0] += rr.y * (double)zz.y;
    }
    for (long long i = 2 * nv + t0; i < n; i += stride) {
        float zi = z32[i];
        if (fixed[i]) {
            zi = 0.f;
            z32[i] = 0.f;
        }
        v[0] += r[i] * (double)zi;
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

// p = z32 + beta p (FP64 direction).
__global__ void k_cgP_p(double *__restrict__ p, const float *__restrict__ z32, long long n, const CGState *st) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    p += zr * n;
    z32 += zr * n;
    st += zr;
    if (st->done) return;
    const double beta = st->beta;
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
    const bool vec = aligned_to(16, p) && aligned_to(8, z32);
    const long long nv = n / 2;
    for (long long i = t0; i < nv; i += stride) {  // pairs of DOFs
        Pair<double> pp = ld_pair(p, i, vec);
        const Pair<float> zz = ld_pair(z32, i, vec);
        pp.x = (double)zz.x + beta * pp.x;
        pp.y = (double)zz.y + beta * pp.y;
        st_pair(p, i, pp, vec);
    }
    for (long long i = 2 * nv + t0; i < n; i += stride) p[i] = (double)z32[i] + beta * p[i];
}

// x = Kinv b on the coarsest level (dense inverse of its operator), one warp per row.
template <typename T>
__global__ void k_dense_mv(const double *__restrict__ K, int n, const T *__restrict__ b, T *__restrict__ x,
                           const CGState *st) {
    const long long zr = blockIdx.z;  // right-hand side of a batched solve (0 otherwise)
    b += zr * n;
    x += zr * n;
    if (st) st += zr;
    if (st && st->done) return;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const double *Kr = K + (long long)row * n;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += Kr[j] * (double)b[j];
    s = warp_sum(s);
    if (lane == 0) x[row] = (T)s;
}

}  // namespace tpo
