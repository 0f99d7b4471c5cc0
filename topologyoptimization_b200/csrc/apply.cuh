// Matrix-free hex8 K*u on the structured grid, node-centric ("owner computes").
//
// Replaces applyAEbe3D / mgApplyA (assembly/index.ts:403-439, 773-817), which loop over
// active elements and scatter-add E_e*Ke*u_e.  Here every thread owns one node column
// (y, z) of the grid and sweeps along x; for each element plane it gathers the 18
// surrounding nodes' values, forms the rows of Ke*u_e that belong to its node for the
// (up to) 8 elements around it, and sums them.  Every output DOF is written exactly
// once: no atomics, no colour passes, and the summation order is fixed.
//
// Element coefficients come from Eact, indexed in z-fastest element order
// (ex*nely + ey)*nelz + ez, holding E_e for active elements and 0 for inactive ones
// (the reference skips elements with E_e <= 1000*Emin).  The hex8 matrix of lk() has
// only kKeClasses distinct values up to sign (ke_pattern.h); the kernel holds those in
// registers and takes each entry's class and sign from the compile-time pattern, so the
// 576 multiply-adds per node need no constant or shared-memory load.
#pragma once
#include "common.cuh"
#include "ke_pattern.h"

namespace tpo {

constexpr int kApplyThreads = 128;

__host__ __device__ inline int apply_rows_e(int nnz) { return (kApplyThreads - 1) / nnz + 3; }
__host__ __device__ inline int apply_np3(int nnz) { return 3 * (kApplyThreads + 2 * nnz + 2); }

constexpr int kApplyStages = 3;  // p / E plane slots: prefetch depth 2

template <typename T>
inline size_t apply_smem_bytes(const Grid &g) {
    return sizeof(T) * (kApplyStages * (size_t)apply_np3(g.nnz) + kApplyStages * (size_t)apply_rows_e(g.nnz) * g.nelz);
}

// Minimum resident CTAs per SM the register budget is sized for: FP64 needs the 54
// doubles of two node planes in registers (3 CTAs); FP32 fits 4.
template <typename T>
struct ApplyOcc {
    static constexpr int value = sizeof(T) == 8 ? 3 : 4;
};

// Epilogue contract:
//   static constexpr int NV;             number of partial sums reduced over the grid
//   void emit(long long dof0, const T acc[3], const T pc[3], double part[NV]);
//   void finalize(const double tot[NV]);  thread 0 of the last block
//   double *partials; unsigned *counter;
//
// Pipeline: plane k+1 of p and plane k of Eact are read from shared memory at the top of
// step k (after one barrier); the copies of p plane k+3 and E plane k+2 are issued into
// the slots that steps k-1/k consumed, so every copy has two steps to land.
// Class values of the element matrix: Ke[i][j] = kKeSign[i*24+j] * v[kKeClass[i*24+j]].
template <typename T>
struct KeCoef {
    T v[kKeClasses];
};

template <typename T>
__device__ __forceinline__ T ke_entry(const T (&kv)[kKeClasses], int idx) {
    return ke_sign(idx) > 0 ? kv[ke_class(idx)] : -kv[ke_class(idx)];
}

template <typename T, class Epi>
__global__ void __launch_bounds__(kApplyThreads, ApplyOcc<T>::value)
k_apply(const __grid_constant__ KeCoef<T> ke, const Grid g, const T *__restrict__ p,
        const T *__restrict__ Eact, const int xchunk, Epi epi, const CGState *__restrict__ st) {
    if (blockIdx.z) {  // right-hand side of a batched solve
        const long long zr = blockIdx.z;
        p += zr * g.ndof;
        if (st) st += zr;
        epi.shift(zr, g.ndof);
    }
    if ((st && st->done) || epi.skip()) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *pbuf = reinterpret_cast<T *>(smem_raw);
    const int NP3 = apply_np3(g.nnz);
    const int NE = apply_rows_e(g.nnz) * g.nelz;
    T *ebuf = pbuf + kApplyStages * NP3;

    const int tid = threadIdx.x;
    const int nnz = g.nnz, nelz = g.nelz;
    const long long ncol = (long long)g.nny * nnz;     // node columns per x-plane
    const long long necol = (long long)g.nely * nelz;  // element columns per x-plane
    const long long c0 = (long long)blockIdx.x * kApplyThreads;
    const long long c = c0 + tid;
    const bool cvalid = c < ncol;
    const int y = cvalid ? (int)(c / nnz) : 0;
    const int z = cvalid ? (int)(c - (long long)y * nnz) : 0;
    const int ylo = (int)(c0 / nnz);
    const long long pbase3 = (c0 - nnz - 1) * 3;        // flat offset of buffer slot 0
    const long long ebase = (long long)(ylo - 1) * nelz;  // flat element offset of slot 0

    const int x0 = blockIdx.y * xchunk;
    const int x1 = min(x0 + xchunk, g.nnx);

    // Buffer positions whose global index lies inside a plane: [plo, phi) and [elo, ehi)
    // (the block-invariant part of the bounds checks, in 32 bits).
    const int plo = (int)max(0LL, -pbase3), phi = (int)min((long long)NP3, ncol * 3 - pbase3);
    const int elo = (int)max(0LL, -ebase), ehi = (int)min((long long)NE, necol - ebase);
    auto load_p = [&](int xk, T *buf) {
        const bool pv = xk >= 0 && xk < g.nnx;
        const T *src = p + (pv ? (long long)xk * ncol * 3 + pbase3 : 0);
        for (int i = tid; i < NP3; i += kApplyThreads) {
            const bool v = pv && i >= plo && i < phi;
            cp_async_elem<T>(buf + i, v ? src + i : p, v);
        }
    };
    auto load_e = [&](int k, T *buf) {
        const bool ev = k >= 0 && k < g.nelx;
        const T *src = Eact + (ev ? (long long)k * necol + ebase : 0);
        for (int i = tid; i < NE; i += kApplyThreads) {
            const bool v = ev && i >= elo && i < ehi;
            cp_async_elem<T>(buf + i, v ? src + i : Eact, v);
        }
    };
    // slot of p plane xk / E plane k within the 3-stage ring (x0-1 -> slot 0)
    auto pslot = [&](int xk) { return pbuf + ((xk - x0 + 1) % kApplyStages) * NP3; };
    auto eslot = [&](int k) { return ebuf + ((k - x0 + 1) % kApplyStages) * NE; };

    T kv[kKeClasses];
#pragma unroll
    for (int i = 0; i < kKeClasses; i++) kv[i] = ke.v[i];
    T PA[3][3][3], PB[3][3][3];
    T accA[3] = {T(0), T(0), T(0)}, accB[3] = {T(0), T(0), T(0)};
    double part[Epi::NV > 0 ? Epi::NV : 1];
#pragma unroll
    for (int k = 0; k < (Epi::NV > 0 ? Epi::NV : 1); k++) part[k] = 0.0;

    // Neighbour values across the z edge of a column belong to elements outside the grid,
    // whose modulus is 0, and positions outside the plane were zero-filled: both are finite
    // and contribute nothing, so no masking is needed here.
    auto read_plane = [&](const T *buf, T (&P)[3][3][3]) {
#pragma unroll
        for (int dy = 0; dy < 3; dy++)
#pragma unroll
            for (int dz = 0; dz < 3; dz++) {
                const int bi = (tid + nnz + 1 + (dy - 1) * nnz + (dz - 1)) * 3;
#pragma unroll
                for (int q = 0; q < 3; q++) P[dy][dz][q] = buf[bi + q];
            }
    };

    // One element-plane step: P0 holds p plane k, P1 receives plane k+1; acc0 is the
    // running sum of node plane k (complete after this step), acc1 starts node plane k+1.
    auto step = [&](int k, T (&P0)[3][3][3], T (&P1)[3][3][3], T (&acc0)[3], T (&acc1)[3]) {
        cp_async_wait_group1();
        __syncthreads();  // p plane k+1 and E plane k have landed; slots of k and k-1 are free
        read_plane(pslot(k + 1), P1);
        T Ee[2][2];
        {
            const T *eb = eslot(k);
#pragma unroll
            for (int ay = 0; ay < 2; ay++)
#pragma unroll
                for (int az = 0; az < 2; az++) {
                    const int ey = y - 1 + ay, ez = z - 1 + az;
                    const bool ok = cvalid && ey >= 0 && ey < g.nely && ez >= 0 && ez < nelz;
                    Ee[ay][az] = ok ? eb[(y - ylo + ay) * nelz + ez] : T(0);
                }
        }
        if (k + 3 <= x1) load_p(k + 3, pslot(k + 3));
        if (k + 2 < x1) load_e(k + 2, eslot(k + 2));
        cp_async_commit();

#pragma unroll
        for (int d = 0; d < 3; d++) acc1[d] = T(0);
#pragma unroll
        for (int ay = 0; ay < 2; ay++)
#pragma unroll
            for (int az = 0; az < 2; az++) {
                const T Ev = Ee[ay][az];
                T u[24];
#pragma unroll
                for (int b = 0; b < 8; b++) {
                    const int bx = (b == 1 || b == 2 || b == 5 || b == 6);
                    const int by = (b == 2 || b == 3 || b == 6 || b == 7);
                    const int bz = (b >= 4);
#pragma unroll
                    for (int q = 0; q < 3; q++) u[b * 3 + q] = bx ? P1[ay + by][az + bz][q] : P0[ay + by][az + bz][q];
                }
                const int L0 = local_node(0, 1 - ay, 1 - az);
                const int L1 = local_node(1, 1 - ay, 1 - az);
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    T s0 = T(0), s1 = T(0);
#pragma unroll
                    for (int j = 0; j < 24; j++) {
                        s0 = fma(ke_entry(kv, (3 * L0 + d) * 24 + j), u[j], s0);
                        s1 = fma(ke_entry(kv, (3 * L1 + d) * 24 + j), u[j], s1);
                    }
                    // an inactive element has Ev = 0, and fma(0, s, acc) = acc for finite s
                    acc0[d] = fma(Ev, s0, acc0[d]);
                    acc1[d] = fma(Ev, s1, acc1[d]);
                }
            }
        if (k >= x0 && cvalid) {
            const long long dof0 = ((long long)k * ncol + c) * 3;
            const T pc[3] = {P0[1][1][0], P0[1][1][1], P0[1][1][2]};
            add_spring(g, dof0, acc0, pc);
            epi.emit(dof0, acc0, pc, part);
        }
    };

    // blocks without planes still take part in the grid reduction below
    if (x0 < x1) {
        // prologue: p planes x0-1, x0, x0+1 and E planes x0-1, x0
        load_p(x0 - 1, pslot(x0 - 1));
        load_p(x0, pslot(x0));
        if (x0 + 1 <= x1) load_p(x0 + 1, pslot(x0 + 1));
        load_e(x0 - 1, eslot(x0 - 1));
        if (x0 < x1) load_e(x0, eslot(x0));
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        read_plane(pslot(x0 - 1), PA);
        for (int k = x0 - 1; k < x1; k++) {
            step(k, PA, PB, accA, accB);
#pragma unroll
            for (int d = 0; d < 3; d++) accA[d] = accB[d];
#pragma unroll
            for (int dy = 0; dy < 3; dy++)
#pragma unroll
                for (int dz = 0; dz < 3; dz++)
#pragma unroll
                    for (int q = 0; q < 3; q++) PA[dy][dz][q] = PB[dy][dz][q];
        }
        cp_async_wait_all();
    }  // x0 < x1

    if constexpr (Epi::NV > 0) {
        __shared__ double sh[32 * Epi::NV];
        double tot[Epi::NV];
        if (grid_sum<Epi::NV>(part, epi.partials, epi.counter, sh, tot)) {
            if (threadIdx.x == 0) epi.finalize(tot);
        }
    }
}

// ---- epilogues -------------------------------------------------------------------
// Every epilogue also names the per-DOF arrays its emit() reads: prefetch(i0, n, t, nt)
// asks L2 for DOFs [i0, i0 + n) of each of them (thread t of nt issues every nt-th line),
// so a kernel can start those reads some plane steps before it emits; pre(i, o) loads one
// node's operands into registers, so a kernel can issue the loads of all its nodes
// before the first store, and emit(i, a, pc, o, part) uses them.  emit(i, a, pc, part)
// does both for one node.

// L2 prefetch of the 128-byte lines that start inside elements [i0, i0 + n) of base.
// Every address issued lies inside the range, so nothing outside the array is touched
// (the partial line at the front is left to the demand load).
template <typename U>
__device__ __forceinline__ void prefetch_l2(const U *base, long long i0, long long n, int t, int nt) {
    if (!base || n <= 0) return;
    const unsigned long long b = reinterpret_cast<unsigned long long>(base + i0);
    const unsigned long long e = reinterpret_cast<unsigned long long>(base + i0 + n);
    for (unsigned long long a = ((b + 127) & ~127ULL) + 128ULL * (unsigned long long)t; a < e;
         a += 128ULL * (unsigned long long)nt)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
}

template <typename T>
struct EpiStore {  // out = K u (optionally zeroed on fixed DOFs)
    static constexpr int NV = 0;
    __device__ bool skip() const { return false; }
    T *out;
    const uint8_t *fixed;  // may be null
    double *partials;
    unsigned *counter;
    // right-hand side z of a batched launch: per-RHS vectors are vs apart
    __device__ void shift(long long z, long long vs) { out += z * vs; }
    __device__ void prefetch(long long i0, long long n, int t, int nt) const { prefetch_l2(fixed, i0, n, t, nt); }
    struct Pre {
        uint8_t fx[3];
    };
    __device__ void pre(long long i, Pre &o) const {
#pragma unroll
        for (int d = 0; d < 3; d++) o.fx[d] = fixed ? fixed[i + d] : 0;
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&)[3], const Pre &o, double *) const {
#pragma unroll
        for (int d = 0; d < 3; d++) out[i + d] = o.fx[d] ? T(0) : a[d];
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&pc)[3], double *part) const {
        Pre o;
        pre(i, o);
        emit(i, a, pc, o, part);
    }
    __device__ void finalize(const double *) const {}
};

template <typename T>
struct EpiSmooth {  // damped Jacobi: xn = x + omega*invD*(b - K x) on free DOFs
    static constexpr int NV = 0;
    __device__ bool skip() const { return false; }
    T *xn;
    const T *b, *invD;
    const uint8_t *fixed;
    T omega;
    double *partials;
    unsigned *counter;
    __device__ void shift(long long z, long long vs) {
        xn += z * vs;
        b += z * vs;
    }
    __device__ void prefetch(long long i0, long long n, int t, int nt) const {
        prefetch_l2(b, i0, n, t, nt);
        prefetch_l2(invD, i0, n, t, nt);
        prefetch_l2(fixed, i0, n, t, nt);
    }
    struct Pre {
        T b[3], invD[3];
        uint8_t fx[3];
    };
    __device__ void pre(long long i, Pre &o) const {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            o.b[d] = b[i + d];
            o.invD[d] = invD[i + d];
            o.fx[d] = fixed[i + d];
        }
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&pc)[3], const Pre &o, double *) const {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const T r = o.b[d] - a[d];
            xn[i + d] = o.fx[d] ? pc[d] : pc[d] + omega * o.invD[d] * r;
        }
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&pc)[3], double *part) const {
        Pre o;
        pre(i, o);
        emit(i, a, pc, o, part);
    }
    __device__ void finalize(const double *) const {}
};

template <typename T>
struct EpiResidual {  // res = b - K x on free DOFs, 0 on fixed
    static constexpr int NV = 0;
    __device__ bool skip() const { return false; }
    T *res;
    const T *b;
    const uint8_t *fixed;
    double *partials;
    unsigned *counter;
    __device__ void shift(long long z, long long vs) {
        res += z * vs;
        b += z * vs;
    }
    __device__ void prefetch(long long i0, long long n, int t, int nt) const {
        prefetch_l2(b, i0, n, t, nt);
        prefetch_l2(fixed, i0, n, t, nt);
    }
    struct Pre {
        T b[3];
        uint8_t fx[3];
    };
    __device__ void pre(long long i, Pre &o) const {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            o.b[d] = b[i + d];
            o.fx[d] = fixed[i + d];
        }
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&)[3], const Pre &o, double *) const {
#pragma unroll
        for (int d = 0; d < 3; d++) res[i + d] = o.fx[d] ? T(0) : o.b[d] - a[d];
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&pc)[3], double *part) const {
        Pre o;
        pre(i, o);
        emit(i, a, pc, o, part);
    }
    __device__ void finalize(const double *) const {}
};

// PCG: Ap = mask(K p), pAp accumulated in FP64; the last block forms alpha.
template <typename T>
struct EpiCG {
    static constexpr int NV = 1;
    __device__ bool skip() const { return false; }
    T *Ap;
    const uint8_t *fixed;
    CGState *st;
    double *partials;
    unsigned *counter;
    __device__ void shift(long long z, long long vs) {
        Ap += z * vs;
        st += z;
        counter = reinterpret_cast<unsigned *>(reinterpret_cast<char *>(counter) + z * (long long)sizeof(CGState));
    }
    __device__ void prefetch(long long i0, long long n, int t, int nt) const { prefetch_l2(fixed, i0, n, t, nt); }
    struct Pre {
        uint8_t fx[3];
    };
    __device__ void pre(long long i, Pre &o) const {
#pragma unroll
        for (int d = 0; d < 3; d++) o.fx[d] = fixed[i + d];
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&pc)[3], const Pre &o, double *part) const {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const T v = o.fx[d] ? T(0) : a[d];
            Ap[i + d] = v;
            part[0] += (double)pc[d] * (double)v;
        }
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&pc)[3], double *part) const {
        Pre o;
        pre(i, o);
        emit(i, a, pc, o, part);
    }
    __device__ void finalize(const double *tot) const {
        st->pAp = tot[0];
        if (st->eps > 0.0) {
            st->alpha = st->rz / (tot[0] + st->eps);
        } else if (tot[0] > 0.0) {
            st->alpha = st->rz / tot[0];
        } else {  // breakdown of the guarded variant: stop with the current iterate
            st->alpha = 0.0;
            st->done = 1;
            st->iters = st->it;
        }
        if (!isfinite(st->alpha)) {
            st->nonfinite = 1;
            st->done = 1;
            st->iters = st->it;
        }
    }
};

// Mixed-precision defect (the reliable update): r = F - K U on free DOFs in FP64, its
// FP32 copy for the inner recurrence, ||r||^2.  Runs only when the gate state asks for an
// update (or when gate is null); then it restarts the FP32 residual from the true one and
// takes the convergence decision on the true FP64 residual.
struct EpiDefect {
    static constexpr int NV = 1;
    double *r;
    float *r32;
    const double *F;
    const uint8_t *fixed;
    CGState *st;
    double *partials;
    unsigned *counter;
    __device__ void shift(long long z, long long vs) {
        r += z * vs;
        r32 += z * vs;
        F += z * vs;
        st += z;
        counter = reinterpret_cast<unsigned *>(reinterpret_cast<char *>(counter) + z * (long long)sizeof(CGState));
    }
    __device__ bool skip() const { return st->done || !st->do_update; }
    __device__ void prefetch(long long i0, long long n, int t, int nt) const {
        prefetch_l2(F, i0, n, t, nt);
        prefetch_l2(fixed, i0, n, t, nt);
    }
    struct Pre {
        double F[3];
        uint8_t fx[3];
    };
    __device__ void pre(long long i, Pre &o) const {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            o.F[d] = F[i + d];
            o.fx[d] = fixed[i + d];
        }
    }
    __device__ void emit(long long i, const double (&a)[3], const double (&)[3], const Pre &o, double *part) const {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double v = o.fx[d] ? 0.0 : o.F[d] - a[d];
            r[i + d] = v;
            r32[i + d] = (float)v;
            part[0] += v * v;
        }
    }
    __device__ void emit(long long i, const double (&a)[3], const double (&pc)[3], double *part) const {
        Pre o;
        pre(i, o);
        emit(i, a, pc, o, part);
    }
    __device__ void finalize(const double *tot) const {
        const double rr = tot[0];
        st->rr = rr;
        if (st->n_updates == 0) {  // tolSq holds tol until the initial residual is known
            st->r0 = rr;
            st->tolSq = st->tolSq * st->tolSq * (rr > 1e-30 ? rr : 1e-30);
        }
        st->maxr2 = rr;
        st->n_updates += 1;
        st->do_update = 0;
        if (!isfinite(rr)) {
            st->nonfinite = 1;
            st->done = 1;
            st->iters = st->it;
        } else if (rr < st->tolSq) {
            st->done = 1;
            st->converged = 1;
            st->iters = st->it;
        } else if (st->it >= st->maxIter) {
            st->done = 1;
            st->iters = st->maxIter;
        }
    }
};

}  // namespace tpo
