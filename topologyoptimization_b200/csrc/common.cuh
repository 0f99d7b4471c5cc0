// Shared device helpers for libtpo (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace tpo {

constexpr int kMaxLevels = 12;

// 24x24 element matrix passed by value as a __grid_constant__ kernel parameter:
// it lives in the constant bank, so warp-uniform indices cost no load instruction.
template <typename T>
struct KeParam {
    T v[576];
};

// Structured grid of unit hex8 elements.  Node n = x*nny*nnz + y*nnz + z (z fastest).
struct Grid {
    int nelx, nely, nelz;
    int nnx, nny, nnz;
    long long nel, nnodes, ndof;
    // optional grounded spring k at one DOF (fine level only): K + k e_sdof e_sdof^T
    long long sdof;
    double sk;
    // x-chunk counts of the structured apply chosen by measurement (FP32, FP64); 0: the
    // launch-shape cost model decides
    int nch[2];
};

// _powDensity (js/optimizer-worker-3d.js:293-306)
__device__ __forceinline__ double pow_density(double x, double p, int intpow) {
    if (intpow && p == floor(p) && p >= 0 && p <= 6) {
        switch ((int)p) {
        case 0: return 1.0;
        case 1: return x;
        case 2: return x * x;
        case 3: return x * x * x;
        case 4: { const double x2 = x * x; return x2 * x2; }
        case 5: { const double x2 = x * x; return x2 * x2 * x; }
        default: { const double x2 = x * x; return x2 * x2 * x2; }
        }
    }
    return pow(x, p);
}

// E = Emin + x^p (E0 - Emin) rounded as the reference rounds it: the product, then the
// sum, never fused into one multiply-add (files built with contraction would otherwise
// fuse them and move E by an ulp).
__device__ __forceinline__ double simp_modulus(double x, double p, double E0, double Emin, int intpow) {
    return __dadd_rn(Emin, __dmul_rn(pow_density(x, p, intpow), E0 - Emin));
}

// acc += k p at the spring DOF when it lies in [dof0, dof0 + 3).
template <typename T>
__device__ __forceinline__ void add_spring(const Grid &g, long long dof0, T (&acc)[3], const T (&pc)[3]) {
    if ((unsigned long long)(g.sdof - dof0) >= 3ULL) return;  // also when sdof < 0 (no spring)
#pragma unroll
    for (int d = 0; d < 3; d++)
        if (dof0 + d == g.sdof) acc[d] = acc[d] + (T)g.sk * pc[d];
}

inline Grid make_grid(int nelx, int nely, int nelz) {
    Grid g;
    g.nelx = nelx; g.nely = nely; g.nelz = nelz;
    g.nnx = nelx + 1; g.nny = nely + 1; g.nnz = nelz + 1;
    g.nel = (long long)nelx * nely * nelz;
    g.nnodes = (long long)g.nnx * g.nny * g.nnz;
    g.ndof = 3 * g.nnodes;
    g.sdof = -1;
    g.sk = 0.0;
    g.nch[0] = g.nch[1] = 0;
    return g;
}

// Scalars of one PCG solve, resident in device memory so that no iteration needs a
// host round trip.  Kernels of an iteration return at once when done != 0.
struct CGState {
    double rz, rz_new, pAp, alpha, beta, rr, r0, tolSq;
    double eps;          // 1e-12 (reference) or 0
    int it;              // iterations completed
    int done;            // solve finished (converged or capped)
    int iters;           // reference-convention iteration count
    int converged;
    int maxIter;
    int nonfinite;
    // mixed precision with reliable updates: the FP32 recursive residual ||r32||^2,
    // the true FP64 ||r||^2 at the last update, the drop factor that triggers the next
    // one, and the trigger itself
    double rr32, maxr2, delta2;
    int do_update, n_updates;
    unsigned int counters[8];
};

// Convergence decision after an iteration that produced ||r||^2 in st->rr, with the
// reference's semantics (tolSq test at the top of the next iteration; cap -> maxIter).
__device__ __forceinline__ void cg_decide(CGState *st) {
    st->it += 1;
    if (!isfinite(st->rr)) {
        st->nonfinite = 1;
        st->done = 1;
        st->iters = st->it;
    } else if (st->rr < st->tolSq) {
        st->done = 1;
        st->converged = 1;
        st->iters = st->it;
    } else if (st->it >= st->maxIter) {
        st->done = 1;
        st->iters = st->maxIter;
    }
}

// True when every pointer is aligned to `a` bytes (the 16-byte vector paths of the
// vector kernels; a batched right-hand side at an odd offset takes the scalar path).
__device__ __forceinline__ bool aligned_to(unsigned a, const void *p0, const void *p1 = nullptr,
                                           const void *p2 = nullptr, const void *p3 = nullptr) {
    const unsigned long long m = (unsigned long long)a - 1ULL;
    return ((reinterpret_cast<unsigned long long>(p0) | reinterpret_cast<unsigned long long>(p1) |
             reinterpret_cast<unsigned long long>(p2) | reinterpret_cast<unsigned long long>(p3)) & m) == 0;
}

// Elements 2i and 2i+1 as one 16-byte (double) or 8-byte (float) access when `vec`, else
// as two scalar accesses: the vector kernels visit DOFs in the same pairs either way, so
// their per-thread sums do not depend on the alignment of a batched right-hand side.
template <typename T>
struct Pair {
    T x, y;
};
template <typename T>
__device__ __forceinline__ Pair<T> ld_pair(const T *a, long long i, bool vec) {
    using V = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    if (vec) {
        const V v = reinterpret_cast<const V *>(a)[i];
        return {(T)v.x, (T)v.y};
    }
    return {a[2 * i], a[2 * i + 1]};
}
template <typename T>
__device__ __forceinline__ void st_pair(T *a, long long i, Pair<T> v, bool vec) {
    using V = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    if (vec) {
        V w;
        w.x = v.x;
        w.y = v.y;
        reinterpret_cast<V *>(a)[i] = w;
    } else {
        a[2 * i] = v.x;
        a[2 * i + 1] = v.y;
    }
}

// ---- reductions --------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Deterministic block sum: fixed warp-shuffle tree, then warp 0 over the warp sums.
// Returns the total in thread 0.  blockDim.x must be a multiple of 32 and <= 1024.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sh /* >= 32*NV */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) sh[k * 32 + wid] = v[k];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double t = lane < nw ? sh[k * 32 + lane] : 0.0;
            v[k] = warp_sum(t);
        }
    }
}

// "Last block finishes" pattern: every block writes its partials, the last block to
// arrive sums all partials in block order (deterministic) and runs the finaliser.
// Returns true in exactly one block, after which partials[0..NV) hold the totals
// (valid in thread 0 only through the out array).
template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double *partials, unsigned int *counter,
                                         double *sh, double (&tot)[NV]) {
    block_sum<NV>(v, sh);
    // one reduction per z-slice of the grid (the right-hand sides of a batched solve)
    const int nb = gridDim.x * gridDim.y;
    const int bid = blockIdx.x + gridDim.x * blockIdx.y;
    partials += (size_t)blockIdx.z * NV * nb;
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) partials[(size_t)k * nb + bid] = v[k];
        __threadfence();
        const unsigned int t = atomicAdd(counter, 1u);
        s_last = (t == (unsigned int)nb - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) acc[k] = 0.0;
    // fixed-order strided sum, then the deterministic block tree
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
#pragma unroll
        for (int k = 0; k < NV; k++) acc[k] += __ldcg(&partials[(size_t)k * nb + i]);
    }
    block_sum<NV>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) tot[k] = acc[k];
        *counter = 0u;  // re-arm for the next launch
    }
    return true;
}

// ---- cp.async (8-byte and 4-byte), zero fill when src_bytes == 0 --------------
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
// 16-byte copy (both addresses 16-byte aligned), cached in L2 only
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }
__device__ __forceinline__ void cp_async_wait_group1() { asm volatile("cp.async.wait_group 1;\n" ::); }
// wait until at most N of this thread's committed cp.async groups are still pending
template <int N>
__device__ __forceinline__ void cp_async_wait_pending() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <typename T>
__device__ __forceinline__ void cp_async_elem(T *smem, const T *gmem, bool valid);
template <>
__device__ __forceinline__ void cp_async_elem<double>(double *s, const double *g, bool v) { cp_async8(s, g, v); }
template <>
__device__ __forceinline__ void cp_async_elem<float>(float *s, const float *g, bool v) { cp_async4(s, g, v); }

// Local index (0..7) of the corner at offset (ox, oy, oz) in {0,1}^3 of a hex8, in the
// reference's local order (0,0,0),(1,0,0),(1,1,0),(0,1,0),(0,0,1),(1,0,1),(1,1,1),(0,1,1).
__host__ __device__ constexpr int local_node(int ox, int oy, int oz) {
    return oz * 4 + (oy ? (ox ? 2 : 3) : (ox ? 1 : 0));
}

// Coordinates of node n (z fastest), in 32-bit arithmetic when the grid allows it.
__device__ __forceinline__ void node_xyz(const Grid &g, long long n, int &x, int &y, int &z) {
    if (g.nnodes < (1LL << 31)) {
        const unsigned u = (unsigned)n, nz = (unsigned)g.nnz, ny = (unsigned)g.nny;
        const unsigned r = u / nz;
        z = (int)(u - r * nz);
        y = (int)(r % ny);
        x = (int)(r / ny);
    } else {
        z = (int)(n % g.nnz);
        const long long r = n / g.nnz;
        y = (int)(r % g.nny);
        x = (int)(r / g.nny);
    }
}

// ---- reference transfer weights (assembly/index.ts:881-969, :983-1042) ----------
// Fine index f maps to c0 = min(f>>1, nC-1) with weight 1-t and c1 = min(c0+1, nC-1)
// with weight t, where t = 0.5 iff c0 != c1 and f is odd.
__host__ __device__ __forceinline__ double w1d(int f, int c, int nC) {
    const int c0 = min(f >> 1, nC - 1);
    const int c1 = min(c0 + 1, nC - 1);
    const double t = (c0 != c1 && (f & 1)) ? 0.5 : 0.0;
    if (c0 == c) return 1.0 - t;
    if (c1 == c && t > 0.0) return t;
    return 0.0;
}

}  // namespace tpo
