// Epilogues of the structured apply kernels (apply_walsh.cuh, apply_tc.cuh).
//
// An apply kernel forms the rows of K*u that belong to one node and hands them to its
// epilogue, which fuses what the solver does next with those rows: store them (applyA,
// assembly/index.ts:403-439), a damped-Jacobi sweep or a residual of the multigrid
// smoother (mgSmooth / mgResidual, assembly/index.ts:837-1048), the PCG operator with its
// p.Ap reduction, or the FP64 defect of the mixed-precision solve.
//
// Epilogue contract:
//   static constexpr int NV;             number of partial sums reduced over the grid
//   bool skip();                         the whole launch has nothing to do
//   void shift(long long z, long long vs); move to right-hand side z of a batched launch
//   void prefetch(i0, n, t, nt);         L2 prefetch of the operands of DOFs [i0, i0 + n)
//   struct Pre; void pre(i, Pre &);      load one node's operands into registers
//   void emit(long long dof0, const T acc[3], const T pc[3], [const Pre &,] double part[NV]);
//   void finalize(const double tot[NV]);  thread 0 of the last block
//   double *partials; unsigned *counter;
#pragma once
#include "common.cuh"

namespace tpo {

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
// prefetch_l2 of DOFs [i0, i0 + n) of several arrays (a null one is skipped): the threads
// split into one group of whole warps per array, at most four warps each (a node plane of
// a tile spans at most 96 lines of an array: one per thread), so that each thread works
// out the line range of a single array and the other warps skip the prefetch.
template <typename... U>
__device__ __forceinline__ void prefetch_split(long long i0, long long n, int t, int nt, const U *...a) {
    constexpr int na = sizeof...(U);
    const int q = min(128, max(32, (nt / na) & ~31));
    const int j = t / q, u = t - j * q;
    int k = 0;
    ((k++ == j ? prefetch_l2(a, i0, n, u, q) : void()), ...);
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
    __device__ void prefetch(long long i0, long long n, int t, int nt) const { prefetch_split(i0, n, t, nt, fixed); }
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
        prefetch_split(i0, n, t, nt, b, invD, fixed);
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

// Chebyshev smoothing sweep k >= 1: x_{k+1} = x_k + cd (x_k - x_{k-1}) + cr D^-1 (b - A x_k)
// on free DOFs (the three-term recurrence of the Chebyshev polynomial smoother, Adams,
// Brezina, Hu, Tuminaro 2003).  x_{k-1} is the old content of the output buffer (the
// V-cycle's sweeps ping-pong between two buffers), read before it is overwritten; with
// xold_zero it is the implicit zero start of a pre-smoothing sequence.
template <typename T>
struct EpiCheb {
    static constexpr int NV = 0;
    __device__ bool skip() const { return false; }
    T *xn;
    const T *b, *invD;
    const uint8_t *fixed;
    T cd, cr;
    int xold_zero;
    double *partials;
    unsigned *counter;
    __device__ void shift(long long z, long long vs) {
        xn += z * vs;
        b += z * vs;
    }
    __device__ void prefetch(long long i0, long long n, int t, int nt) const {
        prefetch_split(i0, n, t, nt, b, invD, fixed, xold_zero ? static_cast<const T *>(nullptr) : xn);
    }
    struct Pre {
        T b[3], invD[3], xo[3];
        uint8_t fx[3];
    };
    // x_{k-1} is read here with the other operands, before any store of the launch: each
    // DOF is read and then overwritten by the same thread
    __device__ void pre(long long i, Pre &o) const {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            o.b[d] = b[i + d];
            o.invD[d] = invD[i + d];
            o.fx[d] = fixed[i + d];
            o.xo[d] = xold_zero ? T(0) : xn[i + d];
        }
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&pc)[3], const Pre &o, double *) const {
#pragma unroll
        for (int d = 0; d < 3; d++)
            xn[i + d] = o.fx[d] ? pc[d] : pc[d] + cd * (pc[d] - o.xo[d]) + cr * o.invD[d] * (o.b[d] - a[d]);
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&pc)[3], double *part) const {
        Pre o;
        pre(i, o);
        emit(i, a, pc, o, part);
    }
    __device__ void finalize(const double *) const {}
};

// The last damped-Jacobi sweep of a preconditioner V-cycle fused with the PCG step that
// follows it: z = xn (0 on fixed DOFs), rz_new = r.z in FP64 over the grid, then beta and
// rz as k_cgP_rz / k_cg_rz form them.
template <typename T>
struct EpiSmoothDot {
    static constexpr int NV = 1;
    __device__ bool skip() const { return false; }
    T *xn;
    const T *b, *invD;
    const uint8_t *fixed;
    T omega;
    const double *r;  // the FP64 PCG residual
    CGState *st;
    double *partials;
    unsigned *counter;
    __device__ void shift(long long z, long long vs) {
        xn += z * vs;
        b += z * vs;
        r += z * vs;
        st += z;
        counter = reinterpret_cast<unsigned *>(reinterpret_cast<char *>(counter) + z * (long long)sizeof(CGState));
    }
    __device__ void prefetch(long long i0, long long n, int t, int nt) const {
        prefetch_split(i0, n, t, nt, b, invD, fixed, r);
    }
    struct Pre {
        T b[3], invD[3];
        double r[3];
        uint8_t fx[3];
    };
    __device__ void pre(long long i, Pre &o) const {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            o.b[d] = b[i + d];
            o.invD[d] = invD[i + d];
            o.r[d] = r[i + d];
            o.fx[d] = fixed[i + d];
        }
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&pc)[3], const Pre &o, double *part) const {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const T z = o.fx[d] ? T(0) : pc[d] + omega * o.invD[d] * (o.b[d] - a[d]);
            xn[i + d] = z;
            part[0] += o.r[d] * (double)z;
        }
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&pc)[3], double *part) const {
        Pre o;
        pre(i, o);
        emit(i, a, pc, o, part);
    }
    __device__ void finalize(const double *tot) const {
        st->rz_new = tot[0];
        if (st->eps > 0.0) st->beta = tot[0] / (st->rz + st->eps);
        else st->beta = st->rz > 0.0 ? tot[0] / st->rz : 0.0;
        st->rz = tot[0];
    }
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
        prefetch_split(i0, n, t, nt, b, fixed);
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
    __device__ void prefetch(long long i0, long long n, int t, int nt) const { prefetch_split(i0, n, t, nt, fixed); }
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

// The coarse step of the reference's "BDDC" preconditioner (bddcApply step 3-4,
// assembly/index.ts:1322-1352): z = x + invD (b - K x) on the coarse (subdomain-corner)
// DOFs, z = x elsewhere, 0 on fixed DOFs.
template <typename T>
struct EpiBddcCoarse {
    static constexpr int NV = 0;
    __device__ bool skip() const { return false; }
    T *out;
    const T *b, *invD;
    const uint8_t *fixed, *coarse;
    double *partials;
    unsigned *counter;
    __device__ void shift(long long z, long long vs) {
        out += z * vs;
        b += z * vs;
    }
    __device__ void prefetch(long long i0, long long n, int t, int nt) const {
        prefetch_split(i0, n, t, nt, b, invD, fixed, coarse);
    }
    struct Pre {
        T b[3], invD[3];
        uint8_t fx[3], cs[3];
    };
    __device__ void pre(long long i, Pre &o) const {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            o.b[d] = b[i + d];
            o.invD[d] = invD[i + d];
            o.fx[d] = fixed[i + d];
            o.cs[d] = coarse[i + d];
        }
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&pc)[3], const Pre &o, double *) const {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const T cc = o.cs[d] ? o.invD[d] * (o.b[d] - a[d]) : T(0);
            out[i + d] = o.fx[d] ? T(0) : pc[d] + cc;
        }
    }
    __device__ void emit(long long i, const T (&a)[3], const T (&pc)[3], double *part) const {
        Pre o;
        pre(i, o);
        emit(i, a, pc, o, part);
    }
    __device__ void finalize(const double *) const {}
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
        prefetch_split(i0, n, t, nt, F, fixed);
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
