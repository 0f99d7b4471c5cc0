// Matrix-free hex8 K*u in the Walsh basis of the element.
//
// Replaces applyAEbe3D / mgApplyA (assembly/index.ts:403-439, 773-817), which loop over
// active elements and scatter-add E_e*Ke*u_e with the dense 24x24 Ke.
//
// The element matrix of a cube (lk(nu), assembly/index.ts) commutes with the three
// mirror symmetries of the cube.  In the basis of Walsh functions over the 8 corners,
// w_(sigma,c)[b, c'] = delta(c, c') * (-1)^(sigma . b) with sigma, b in {0,1}^3, the
// mirrors are diagonal, so Ke is block diagonal: 8 blocks of 3x3, one per sign pattern
// of the three mirrors.  Those blocks are sparse as well (rigid translations and
// rotations are in their null space; the cube's rotations make two of them circulant), so
// Ke*u_e = W B W^T u_e costs
//   forward transform  48 add/sub (a 2x2x2 butterfly per displacement component),
//   B                  33 flops plus 8 to fold E_e into B's constants (for lk(nu)),
//   inverse transform  48 add/sub,
// about 140 operations instead of 576 multiply-adds.  The sweep along x shares half of
// each transform between neighbouring element planes: a node plane's (y, z) butterfly
// is computed once, and the contributions an element plane makes to the next node plane
// are carried in the (y, z) Walsh domain, so one inverse butterfly per element and step
// finishes both.
//
// Work layout.  Node columns (y, z) of a plane are numbered c = y*nnz + z.  An element is
// named by its base node column e (its corner (0,0)); columns with y = nny-1 or
// z = nnz-1 name no element and carry E = 0.  A CTA owns NT*ME element columns
// [e0, e0 + NEB) and the node columns [e0 + nnz + 1, e0 + NEB) whose four surrounding
// elements it computes (the first nnz + 1 element columns are recomputed by the previous
// CTA: a one-row halo).  It sweeps its x-chunk of node planes: at step k it forms the
// element plane k from node planes k and k+1 and writes each element's contributions to
// the four corners of node plane k into one of two shared exchange buffers; then each
// node of plane k-1, whose corners were written before the step's barrier, sums its four
// (a fixed order: no atomics, bit-reproducible) and hands the row of K*u to the
// epilogue.  One barrier per step.  Node planes arrive by 16-byte cp.async into a 5-slot
// ring (2 planes ahead), element planes into a 3-slot ring.
#pragma once
#include "apply.cuh"

namespace tpo {

// Constants of the Walsh blocks of a cube element matrix.  With v the Walsh coefficients
// of u_e (unnormalised, v = W^T u) the blocks give y = B v with B = W^T Ke W / 64:
//   twist block       y_i = a1 v_i + a2 (v_0 + v_1 + v_2)
//   three shear       y_0 = p v_0 + q v_1, y_1 = q v_0 + p v_1, y_2 = d v_2
//   three bending     y_0 = s v_0, y_1 = e v_1 + f v_2, y_2 = f v_1 + e v_2
//   normal strains    y_i = g1 v_i + g2 (v_0 + v_1 + v_2)
// Every matrix with the cube's symmetries has this form.  For lk(nu) itself p = q (the
// rigid rotation v_0 = -v_1 has no energy) and s = 0 (rigid translation), and the kernel
// instantiated with kGeneral = false uses that; a Ke whose entries were rounded (a
// single-precision KEflat) breaks both by its rounding, and kGeneral = true keeps them.
template <typename T>
struct WalshKe {
    T a1, a2, p, q, d, e, f, s, g1, g2;
    int general;  // p != q or s != 0 beyond double rounding (host-side choice of instantiation)
};

// Threads per CTA, element columns per thread and the CTA's element columns.  A thread
// carries 24 values of transform state per element (48 registers per FP64 element), and
// one CTA of 512 threads runs per SM: FP32 threads take two elements, FP64 threads one.
template <typename T>
struct WTile {
    static constexpr int NT = 512;
    static constexpr int ME = sizeof(T) == 8 ? 1 : 2;
    static constexpr int NEB = ME * NT;  // element columns per CTA
};

__host__ __device__ inline long long floor_div_ll(long long a, long long b) {
    return a >= 0 ? a / b : -((-a + b - 1) / b);
}
template <typename T>
__host__ __device__ inline int walsh_out_cols(int nnz) { return WTile<T>::NEB - nnz - 1; }
template <typename T>
__host__ __device__ inline int walsh_np3(int nnz) { return 3 * (WTile<T>::NEB + nnz + 1); }
template <typename T>
__host__ __device__ inline int walsh_rows_e(int nnz) { return (WTile<T>::NEB - 1) / nnz + 2; }

// Slot size of a slab of n elements: room for the offset of its first element within a
// 16-byte chunk and for the copied chunks.
template <typename T>
__host__ __device__ inline int walsh_slot(int n) {
    constexpr int V = 16 / (int)sizeof(T);
    return (n + 2 * V + V - 1) / V * V;
}

constexpr int kWPStages = 5, kWEStages = 3;

template <typename T>
inline size_t walsh_smem_bytes(const Grid &g) {
    return sizeof(T) * ((size_t)kWPStages * walsh_slot<T>(walsh_np3<T>(g.nnz)) +
                        (size_t)kWEStages * walsh_slot<T>(walsh_rows_e<T>(g.nnz) * g.nelz) + (size_t)24 * WTile<T>::NEB);
}

// Element offset of `first` within its 16-byte chunk.
template <typename T>
__device__ __forceinline__ int chunk_offset(const T *first) {
    return (int)((reinterpret_cast<unsigned long long>(first) & 15ULL) / sizeof(T));
}

// Stage elements [first, first + n) into buf + chunk_offset(first) by 16-byte cp.async of
// the aligned chunks that cover them (thread tid of nt takes every nt-th chunk).  Only
// [lo, hi) is readable: a chunk that crosses either end is copied element by element with
// zero fill outside; valid == false (a plane outside the grid) zero-fills the slab with
// plain stores.  Elements outside the plane but inside [lo, hi) are copied as they are:
// the kernel gives them weight 0.
template <typename T>
__device__ __forceinline__ void stage_slab(T *buf, const T *first, int n, const T *lo, const T *hi, bool valid,
                                           int tid, int nt) {
    constexpr int V = 16 / (int)sizeof(T);
    const int sh = chunk_offset(first);
    const int nch = (sh + n + V - 1) / V;
    if (!valid) {
        for (int j = tid; j < nch; j += nt) reinterpret_cast<uint4 *>(buf)[j] = make_uint4(0u, 0u, 0u, 0u);
        return;
    }
    const unsigned long long ulo = reinterpret_cast<unsigned long long>(lo);
    const unsigned long long uhi = reinterpret_cast<unsigned long long>(hi);
    const unsigned long long base = reinterpret_cast<unsigned long long>(first) - (unsigned long long)sh * sizeof(T);
    for (int j = tid; j < nch; j += nt) {
        const unsigned long long src = base + 16ULL * (unsigned long long)j;
        T *d = buf + j * V;
        if (src >= ulo && src + 16ULL <= uhi) {
            cp_async16(d, reinterpret_cast<const void *>(src));
        } else {
#pragma unroll
            for (int q = 0; q < V; q++) {
                const unsigned long long a = src + (unsigned long long)q * sizeof(T);
                const bool ok = a >= ulo && a < uhi;
                cp_async_elem<T>(d + q, ok ? reinterpret_cast<const T *>(a) : lo, ok);
            }
        }
    }
}

// One node plane's (y, z) butterfly for an element: the 4 corners (by, bz) at node
// columns le, le+1, le+nnz, le+nnz+1 of the slab (a00 = 3 le, a10 = 3 (le + nnz))
// -> h[s][c], s = 2*sigma_y + sigma_z.
template <typename T>
__device__ __forceinline__ void walsh_yz(const T *__restrict__ slab, int a00, int a10, T (&h)[4][3]) {
    const T *p00 = slab + a00;  // 3 * le
    const T *p10 = slab + a10;  // 3 * (le + nnz)
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const T n00 = p00[c], n01 = p00[3 + c], n10 = p10[c], n11 = p10[3 + c];
        const T a = n00 + n01, b = n00 - n01, cc = n10 + n11, d = n10 - n11;
        h[0][c] = a + cc;
        h[1][c] = b + d;
        h[2][c] = a - cc;
        h[3][c] = b - d;
    }
}

// ---- FP32: the thread's two element columns as the lanes of packed f32x2 arithmetic ----
// Blackwell executes add / multiply / fma on a pair of FP32 values held in one 64-bit
// register pair as one instruction.  The FP32 kernel keeps each transform value of its
// two elements (columns le = tid and tid + NT) in such a pair, so every operation of the
// transforms and blocks is issued once for both elements.
struct P2 {
    float2 v;
};
__device__ __forceinline__ P2 operator+(P2 a, P2 b) { return {__fadd2_rn(a.v, b.v)}; }
// a - b as fma(b, -1, a): one rounding, the same value as the subtraction
__device__ __forceinline__ P2 operator-(P2 a, P2 b) { return {__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v)}; }
__device__ __forceinline__ P2 operator*(P2 a, P2 b) { return {__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ P2 pfma(P2 a, P2 b, P2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ P2 splat(float s) { return {make_float2(s, s)}; }

// (y, z) butterfly of one node plane for both elements: corners at slab offsets
// a00[j] (= 3 le_j) and a10[j] (= 3 (le_j + nnz)).
__device__ __forceinline__ void walsh_yz2(const float *__restrict__ slab, const int (&a00)[2], const int (&a10)[2],
                                          P2 (&h)[4][3]) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const P2 n00{make_float2(slab[a00[0] + c], slab[a00[1] + c])};
        const P2 n01{make_float2(slab[a00[0] + 3 + c], slab[a00[1] + 3 + c])};
        const P2 n10{make_float2(slab[a10[0] + c], slab[a10[1] + c])};
        const P2 n11{make_float2(slab[a10[0] + 3 + c], slab[a10[1] + 3 + c])};
        const P2 a = n00 + n01, b = n00 - n01, cc = n10 + n11, d = n10 - n11;
        h[0][c] = a + cc;
        h[1][c] = b + d;
        h[2][c] = a - cc;
        h[3][c] = b - d;
    }
}

// One element step of the FP32 kernel for both elements: x stage of node planes k and
// k+1 (Pw, Qw), the Walsh blocks scaled by E, the inverse x stage, and Z = the (y, z)
// Walsh-domain contributions to node plane k (carry takes those to plane k+1).  The same
// operations as the scalar step of k_apply_w, for lk's block form (kGeneral = false).
__device__ __forceinline__ void walsh_step2(const WalshKe<float> &wk, P2 E, P2 (&Pw)[4][3], const P2 (&Qw)[4][3],
                                            P2 (&carry)[4][3], P2 (&Z)[4][3]) {
    P2 v0[4][3], v1[4][3];
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            v0[s][c] = Pw[s][c] + Qw[s][c];
            v1[s][c] = Pw[s][c] - Qw[s][c];
            Pw[s][c] = Qw[s][c];
        }
    const P2 a1 = E * splat(wk.a1), a2 = E * splat(wk.a2), ps = E * splat(wk.p), ds = E * splat(wk.d);
    const P2 es = E * splat(wk.e), fs = E * splat(wk.f), g1 = E * splat(wk.g1), g2 = E * splat(wk.g2);
    const P2 zero = splat(0.0f);
    {  // twist: (110,z) (101,y) (011,x)
        const P2 t = a2 * ((v1[2][2] + v1[1][1]) + v0[3][0]);
        v1[2][2] = pfma(a1, v1[2][2], t);
        v1[1][1] = pfma(a1, v1[1][1], t);
        v0[3][0] = pfma(a1, v0[3][0], t);
    }
    {  // normal strains: (100,x) (010,y) (001,z)
        const P2 t = g2 * ((v1[0][0] + v0[2][1]) + v0[1][2]);
        v1[0][0] = pfma(g1, v1[0][0], t);
        v0[2][1] = pfma(g1, v0[2][1], t);
        v0[1][2] = pfma(g1, v0[1][2], t);
    }
    {  // shear pairs (p = q): both entries become p (u0 + u1)
        const P2 t0 = ps * (v1[0][1] + v0[2][0]);
        v1[0][1] = t0;
        v0[2][0] = t0;
        const P2 t1 = ps * (v1[0][2] + v0[1][0]);
        v1[0][2] = t1;
        v0[1][0] = t1;
        const P2 t2 = ps * (v0[2][2] + v0[1][1]);
        v0[2][2] = t2;
        v0[1][1] = t2;
        v1[3][2] = ds * v1[3][2];
        v1[3][1] = ds * v1[3][1];
        v1[3][0] = ds * v1[3][0];
    }
    {  // bending: rigid translations (000, *) carry no energy
        v0[0][0] = zero;
        v0[0][1] = zero;
        v0[0][2] = zero;
        P2 pp = v1[2][1], qq = v1[1][2];
        v1[2][1] = pfma(es, pp, fs * qq);
        v1[1][2] = pfma(fs, pp, es * qq);
        pp = v1[2][0];
        qq = v0[3][2];
        v1[2][0] = pfma(es, pp, fs * qq);
        v0[3][2] = pfma(fs, pp, es * qq);
        pp = v1[1][0];
        qq = v0[3][1];
        v1[1][0] = pfma(es, pp, fs * qq);
        v0[3][1] = pfma(fs, pp, es * qq);
    }
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            Z[s][c] = (v0[s][c] + v1[s][c]) + carry[s][c];
            carry[s][c] = v0[s][c] - v1[s][c];
        }
}

template <typename T, class Epi, bool kGeneral>
__global__ void __launch_bounds__(WTile<T>::NT, 1)
k_apply_w(const __grid_constant__ WalshKe<T> wk, const Grid g, const T *__restrict__ p, const T *__restrict__ Eact,
          const int xchunk, Epi epi, const CGState *__restrict__ st) {
    constexpr int ME = WTile<T>::ME, NEB = WTile<T>::NEB, kWThreads = WTile<T>::NT;
    if (blockIdx.z) {  // right-hand side of a batched solve
        const long long zr = blockIdx.z;
        p += zr * g.ndof;
        if (st) st += zr;
        epi.shift(zr, g.ndof);
    }
    if ((st && st->done) || epi.skip()) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nnz = g.nnz, nelz = g.nelz;
    const int NP3 = walsh_np3<T>(nnz);
    const int NER = walsh_rows_e<T>(nnz);
    const int NE = NER * nelz;
    const int TOUT = walsh_out_cols<T>(nnz);
    const int NP3S = walsh_slot<T>(NP3), NES = walsh_slot<T>(NE);
    T *pbuf = reinterpret_cast<T *>(smem_raw);
    T *ebuf = pbuf + kWPStages * NP3S;
    T *xbuf = ebuf + kWEStages * NES;  // 2 x [corner 4][component 3][NEB]: planes k and k-1

    const int tid = threadIdx.x;
    const long long ncol = (long long)g.nny * nnz;     // node columns per x-plane
    const long long necol = (long long)g.nely * nelz;  // elements per x-plane
    const long long c0 = (long long)blockIdx.x * TOUT;  // first output node column
    const long long e0 = c0 - nnz - 1;                  // first element column
    const long long er0 = floor_div_ll(e0, nnz);        // first element row (y) in the E slab
    const long long pg0 = e0 * 3;                       // flat offset of slab slot 0 in a plane
    const long long eg0 = er0 * nelz;                   // flat element offset of E slab slot 0

    const int x0 = blockIdx.y * xchunk;
    const int x1 = min(x0 + xchunk, g.nnx);

    // first element of the node / element slab of a plane (address only: it may lie
    // outside the arrays, whose readable ranges are [p, p + ndof) and [Eact, Eact + nel))
    auto pfirst = [&](int xk) { return p + ((long long)xk * ncol * 3 + pg0); };
    auto efirst = [&](int k) { return Eact + ((long long)k * necol + eg0); };
    auto load_p = [&](int xk, T *buf) {
        stage_slab<T>(buf, pfirst(xk), NP3, p, p + g.ndof, xk >= 0 && xk < g.nnx, tid, kWThreads);
    };
    auto load_e = [&](int k, T *buf) {
        stage_slab<T>(buf, efirst(k), NE, Eact, Eact + g.nel, k >= 0 && k < g.nelx, tid, kWThreads);
    };
    // A staged slab starts at its slot base + the first element's offset within its 16-byte
    // chunk (chunk_offset).  Successive planes' first elements are a fixed stride apart, so
    // the offset of plane xk follows from 32-bit arithmetic on the low address bits.
    const unsigned plo4 = (unsigned)reinterpret_cast<unsigned long long>(pfirst(0));
    const unsigned pst4 = (unsigned)(ncol * 3 * (long long)sizeof(T));
    const unsigned elo4 = (unsigned)reinterpret_cast<unsigned long long>(efirst(0));
    const unsigned est4 = (unsigned)(necol * (long long)sizeof(T));
    constexpr int kLg = sizeof(T) == 8 ? 3 : 2;
    auto poff = [&](int xk) { return (int)(((plo4 + (unsigned)xk * pst4) & 15u) >> kLg); };
    auto eoff = [&](int k) { return (int)(((elo4 + (unsigned)k * est4) & 15u) >> kLg); };

    // this thread's elements: slab offsets of their corners (0,0) and (1,0), E-slab index
    // (-1: no element)
    int eidx[ME], a00[ME], a10[ME];
#pragma unroll
    for (int j = 0; j < ME; j++) {
        const int le = tid + j * kWThreads;
        const long long e = e0 + le;
        const long long y = floor_div_ll(e, nnz);
        const int z = (int)(e - y * nnz);
        eidx[j] = (e >= 0 && y < g.nely && z < nelz) ? (int)((y - er0) * nelz + z) : -1;
        a00[j] = 3 * le;
        a10[j] = 3 * (le + nnz);
    }

    double part[Epi::NV > 0 ? Epi::NV : 1];
#pragma unroll
    for (int k = 0; k < (Epi::NV > 0 ? Epi::NV : 1); k++) part[k] = 0.0;

    // L2 prefetch of the epilogue's operands for this CTA's nodes of plane xk
    const int nout = (int)min((long long)TOUT, ncol - c0);
    auto prefetch_plane = [&](int xk) {
        if (xk >= x0 && xk < x1) epi.prefetch(((long long)xk * ncol + c0) * 3, 3LL * nout, tid, kWThreads);
    };

    T Pw[ME][4][3];     // (y, z) butterfly of node plane k for each element
    T carry[ME][4][3];  // element plane k-1's contributions to node plane k, (y, z) Walsh domain
    // FP32 (lk's block form): the same state for both elements in packed pairs
    constexpr bool kPack = std::is_same_v<T, float> && ME == 2 && !kGeneral;
    P2 Pw2[4][3], carry2[4][3];

    if (x0 < x1) {
        // Ring slots at step k: node planes k-2 (free: receives k+3), k-1, k, k+1, k+2 and
        // element planes k-1 (free: receives k+2), k, k+1; rotated after every step.
        T *sp_f = pbuf + 4 * NP3S, *sp_m = pbuf + 3 * NP3S, *sp_0 = pbuf, *sp_1 = pbuf + NP3S, *sp_2 = pbuf + 2 * NP3S;
        T *se_m = ebuf + 2 * NES, *se_0 = ebuf, *se_1 = ebuf + NES;
        // node phase of plane xk: its four corner sums from the exchange buffer, the
        // epilogue operands loaded before any store
        auto node_phase = [&](int xk, const T *pk, const T *xb) {
            const long long dofk = ((long long)xk * ncol + c0) * 3;
            typename Epi::Pre opnd[ME];
#pragma unroll
            for (int j = 0; j < ME; j++) {
                const int ln = tid + j * kWThreads;
                if (ln < nout) epi.pre(dofk + 3 * ln, opnd[j]);
            }
#pragma unroll
            for (int j = 0; j < ME; j++) {
                const int ln = tid + j * kWThreads;
                if (ln >= nout) break;
                T acc[3], pc[3];
                const T *xn = xb + ln;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    // corner (0,0) of element n, (0,1) of n-1, (1,0) of n-nnz, (1,1) of n-nnz-1
                    acc[c] = ((xn[(0 * 3 + c) * NEB + nnz + 1] + xn[(1 * 3 + c) * NEB + nnz]) + xn[(2 * 3 + c) * NEB + 1]) +
                             xn[(3 * 3 + c) * NEB];
                    pc[c] = pk[3 * (ln + nnz + 1) + c];
                }
                const long long dof0 = dofk + 3 * ln;
                add_spring(g, dof0, acc, pc);
                epi.emit(dof0, acc, pc, opnd[j], part);
            }
        };
        // prologue: node planes x0-1, x0, x0+1 and element planes x0-1, x0
        prefetch_plane(x0);
        prefetch_plane(x0 + 1);
        load_p(x0 - 1, sp_0);
        load_p(x0, sp_1);
        if (x0 + 1 <= x1) load_p(x0 + 1, sp_2);
        load_e(x0 - 1, se_0);
        load_e(x0, se_1);
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        {
            const T *q = sp_0 + poff(x0 - 1);
            if constexpr (kPack) {
                walsh_yz2(q, a00, a10, Pw2);
#pragma unroll
                for (int s = 0; s < 4; s++)
#pragma unroll
                    for (int c = 0; c < 3; c++) carry2[s][c] = splat(0.0f);
            } else {
#pragma unroll
                for (int j = 0; j < ME; j++) {
                    walsh_yz<T>(q, a00[j], a10[j], Pw[j]);
#pragma unroll
                    for (int s = 0; s < 4; s++)
#pragma unroll
                        for (int c = 0; c < 3; c++) carry[j][s][c] = T(0);
                }
            }
        }

        for (int k = x0 - 1; k < x1; k++) {
            cp_async_wait_group1();
            // node plane k+1 and element plane k have landed; step k-1 is done everywhere,
            // so the slots of node plane k-2, element plane k-1 and exchange buffer k-2 are free
            __syncthreads();
            if (k + 3 <= x1) load_p(k + 3, sp_f);
            if (k + 2 < x1) load_e(k + 2, se_m);
            cp_async_commit();
            prefetch_plane(k + 3);

            const T *q = sp_1 + poff(k + 1);
            const T *eb = se_0 + eoff(k);
            const bool emit_plane = k >= x0;
            if constexpr (kPack) {
                const P2 E{make_float2(eidx[0] >= 0 ? eb[eidx[0]] : 0.0f, eidx[1] >= 0 ? eb[eidx[1]] : 0.0f)};
                P2 Qw[4][3], Z[4][3];
                walsh_yz2(q, a00, a10, Qw);
                walsh_step2(wk, E, Pw2, Qw, carry2, Z);
                if (emit_plane) {
                    // inverse (y, z) butterfly -> corners (by, bz) of node plane k, one store per lane
                    T *xo = xbuf + (k & 1) * 12 * NEB + tid;
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const P2 A = Z[0][c] + Z[1][c], B = Z[0][c] - Z[1][c];
                        const P2 C = Z[2][c] + Z[3][c], D = Z[2][c] - Z[3][c];
                        const P2 o0 = A + C, o1 = B + D, o2 = A - C, o3 = B - D;
                        xo[(0 * 3 + c) * NEB] = o0.v.x;
                        xo[(0 * 3 + c) * NEB + kWThreads] = o0.v.y;
                        xo[(1 * 3 + c) * NEB] = o1.v.x;
                        xo[(1 * 3 + c) * NEB + kWThreads] = o1.v.y;
                        xo[(2 * 3 + c) * NEB] = o2.v.x;
                        xo[(2 * 3 + c) * NEB + kWThreads] = o2.v.y;
                        xo[(3 * 3 + c) * NEB] = o3.v.x;
                        xo[(3 * 3 + c) * NEB + kWThreads] = o3.v.y;
                    }
                }
            } else
#pragma unroll
            for (int j = 0; j < ME; j++) {
                const int le = tid + j * kWThreads;
                const T E = eidx[j] >= 0 ? eb[eidx[j]] : T(0);
                T Qw[4][3];
                walsh_yz<T>(q, a00[j], a10[j], Qw);
                // x stage: v0 = sigma_x 0, v1 = sigma_x 1
                T v0[4][3], v1[4][3];
#pragma unroll
                for (int s = 0; s < 4; s++)
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        v0[s][c] = Pw[j][s][c] + Qw[s][c];
                        v1[s][c] = Pw[j][s][c] - Qw[s][c];
                        Pw[j][s][c] = Qw[s][c];
                    }
                // blocks, E folded into the constants (y overwrites v in place)
                const T a1 = E * wk.a1, a2 = E * wk.a2, ps = E * wk.p, ds = E * wk.d;
                const T es = E * wk.e, fs = E * wk.f, g1 = E * wk.g1, g2 = E * wk.g2;
                const T qs = kGeneral ? E * wk.q : ps, ss = kGeneral ? E * wk.s : T(0);
                // shear pair (v_0, v_1) -> (p v_0 + q v_1, q v_0 + p v_1)
                auto shear = [&](T &u0, T &u1) {
                    if constexpr (kGeneral) {
                        const T w0 = u0, w1 = u1;
                        u0 = fma(ps, w0, qs * w1);
                        u1 = fma(qs, w0, ps * w1);
                    } else {
                        const T t = ps * (u0 + u1);
                        u0 = t;
                        u1 = t;
                    }
                };
                auto rigid = [&](T &u) { u = kGeneral ? ss * u : T(0); };
                {  // twist: (110,z) (101,y) (011,x)
                    const T t = a2 * (v1[2][2] + v1[1][1] + v0[3][0]);
                    v1[2][2] = fma(a1, v1[2][2], t);
                    v1[1][1] = fma(a1, v1[1][1], t);
                    v0[3][0] = fma(a1, v0[3][0], t);
                }
                {  // normal strains: (100,x) (010,y) (001,z)
                    const T t = g2 * (v1[0][0] + v0[2][1] + v0[1][2]);
                    v1[0][0] = fma(g1, v1[0][0], t);
                    v0[2][1] = fma(g1, v0[2][1], t);
                    v0[1][2] = fma(g1, v0[1][2], t);
                }
                // shear xy: (100,y) (010,x) | (111,z)
                shear(v1[0][1], v0[2][0]);
                v1[3][2] = ds * v1[3][2];
                // shear xz: (100,z) (001,x) | (111,y)
                shear(v1[0][2], v0[1][0]);
                v1[3][1] = ds * v1[3][1];
                // shear yz: (010,z) (001,y) | (111,x)
                shear(v0[2][2], v0[1][1]);
                v1[3][0] = ds * v1[3][0];
                {  // bending about x: (000,x) rigid | (110,y) (101,z)
                    const T pp = v1[2][1], qq = v1[1][2];
                    rigid(v0[0][0]);
                    v1[2][1] = fma(es, pp, fs * qq);
                    v1[1][2] = fma(fs, pp, es * qq);
                }
                {  // bending about y: (000,y) rigid | (110,x) (011,z)
                    const T pp = v1[2][0], qq = v0[3][2];
                    rigid(v0[0][1]);
                    v1[2][0] = fma(es, pp, fs * qq);
                    v0[3][2] = fma(fs, pp, es * qq);
                }
                {  // bending about z: (000,z) rigid | (101,x) (011,y)
                    const T pp = v1[1][0], qq = v0[3][1];
                    rigid(v0[0][2]);
                    v1[1][0] = fma(es, pp, fs * qq);
                    v0[3][1] = fma(fs, pp, es * qq);
                }
                // inverse x stage: node plane k gets y0 + y1 (plus the carry), k+1 gets y0 - y1
                T Z[4][3];
#pragma unroll
                for (int s = 0; s < 4; s++)
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        Z[s][c] = (v0[s][c] + v1[s][c]) + carry[j][s][c];
                        carry[j][s][c] = v0[s][c] - v1[s][c];
                    }
                if (emit_plane) {
                    // inverse (y, z) butterfly -> corners (by, bz) of node plane k
                    T *xo = xbuf + (k & 1) * 12 * NEB + le;
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const T A = Z[0][c] + Z[1][c], B = Z[0][c] - Z[1][c];
                        const T C = Z[2][c] + Z[3][c], D = Z[2][c] - Z[3][c];
                        xo[(0 * 3 + c) * NEB] = A + C;  // (0,0)
                        xo[(1 * 3 + c) * NEB] = B + D;  // (0,1)
                        xo[(2 * 3 + c) * NEB] = A - C;  // (1,0)
                        xo[(3 * 3 + c) * NEB] = B - D;  // (1,1)
                    }
                }
            }

            // node plane k-1: every element of plane k-1 wrote its corners before the barrier
            if (k - 1 >= x0) node_phase(k - 1, sp_m + poff(k - 1), xbuf + ((k - 1) & 1) * 12 * NEB);
            // rotate the rings
            T *t = sp_f;
            sp_f = sp_m;
            sp_m = sp_0;
            sp_0 = sp_1;
            sp_1 = sp_2;
            sp_2 = t;
            t = se_m;
            se_m = se_0;
            se_0 = se_1;
            se_1 = t;
        }
        __syncthreads();  // the last plane's corners
        node_phase(x1 - 1, sp_m + poff(x1 - 1), xbuf + ((x1 - 1) & 1) * 12 * NEB);
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

}  // namespace tpo
