// Tensor-core element contraction for the FP32 K*u of the mixed-precision solves.
//
// For every element plane the products Y_e = Ke * (E_e u_e) of the 256 elements of a tile
// run as tcgen05.mma of shape M=128 (elements) x N=32 (24 outputs + 8 zero rows of Ke) x
// K=24 (u_e), A and B staged in shared memory in the canonical no-swizzle K-major
// core-matrix layout, the FP32 accumulator in tensor memory.  Operand modes (kMode):
//   0  TF32 operands (kind::tf32, K = 8 per MMA, 3 MMAs);
//   1  3xTF32: the operands split into TF32 high and low parts and D = Ah*Bh + Ah*Bl +
//      Al*Bh, which restores FP32-class accuracy;
//   2  BF16 operands (kind::f16, K = 16 per MMA, K padded to 32 with zeros, 2 MMAs):
//      half the operand bytes of TF32 and an 8-bit mantissa.  One thread per element reads its 24 outputs back with
// tcgen05.ld; node sums come from a warp shuffle along z (lanes are z-consecutive
// elements) and one shared-memory exchange along y (warps are y-consecutive element
// rows).  Nodes own their sum, as in k_apply: no atomics.
//
// CTA: 256 threads = 8 element rows x 32 elements; it owns the 7 x 31 nodes whose four
// (y,z)-adjacent elements all lie in the tile (tiles overlap by one element row/column)
// and sweeps an x-chunk, carrying the plane-k+1 partial sums.  Pipeline per element
// plane k: wait for node plane k+1 and for MMA(k-1) | prefetch node plane k+2 | build
// A(k) | issue MMA(k) into tensor-memory stage k%2 | epilogue of plane k-1 from stage
// (k-1)%2 while MMA(k) runs.
//
// Every mbarrier wait is bounded; on expiry the kernel records the failure in *err,
// stops issuing work, waits (bounded) for its last MMA, releases its tensor memory and
// returns.
#pragma once
#include "apply.cuh"

namespace tpo {

constexpr int kTcThreads = 256;
constexpr int kTcRowsE = 8;   // element rows per tile (y)
constexpr int kTcColsE = 32;  // elements per row (z)
constexpr int kTcNodesY = kTcRowsE - 1;
constexpr int kTcNodesZ = kTcColsE - 1;
constexpr int kTcPRow = (kTcColsE + 1) * 3;           // floats per staged node row (99)
constexpr int kTcPPlane = (kTcRowsE + 1) * kTcPRow;   // floats per staged node plane (891)
constexpr int kTcPSlot = 896;                         // padded ring slot
// node-plane ring: planes k, k+1 in use, k+2 .. k+R-1 landing (R-2 planes of lead)
__host__ __device__ constexpr int tc_ring(bool split) { return split ? 4 : 5; }
constexpr int kTcLoads = (kTcPPlane + kTcThreads - 1) / kTcThreads;
constexpr int kTcMBlock = 128 * 24 * 4;               // bytes of one M=128 operand block (TF32)
constexpr int kTcATile = 2 * kTcMBlock;               // 256 elements
constexpr int kTcBTile = 32 * 24 * 4;                 // bytes of a B tile (32 rows x 24 tf32)
constexpr int kTcMBlockBf = 128 * 32 * 2;             // BF16: 128 rows x 32 (24 + 8 zero) values
constexpr int kTcBTileBf = 32 * 32 * 2;
constexpr int kTcXch = kTcThreads * 6;                // floats of the y-exchange buffer
constexpr uint32_t kTcCols = 128;                     // 2 stages x 2 blocks x 32 columns
constexpr long long kTcWaitCycles = 2000000000LL;     // about one second at B200 clocks

// Ke^T as the B operand, row n (output) = Ke row n for n < 24, zero rows 24..31; high and
// low TF32 parts (hi = rna(Ke), lo = rna(Ke - hi)) and the BF16 rounding (nearest even,
// K padded to 32 with zeros), already in core-matrix order.
struct TcKe {
    float bhi[32 * 24];
    float blo[32 * 24];
    uint16_t bbf[32 * 32];
};

// Byte offset of element (row r, k-chunk c of 4 values) in a K-major no-swizzle tile
// with 24 values per row: 8-row core matrices of 16-byte rows; the 6 chunks of one
// 8-row group are adjacent (LBO = 128 B) and groups are 768 B apart (SBO).
__host__ __device__ constexpr int tc_core_offset(int r, int c) { return (r >> 3) * 768 + c * 128 + (r & 7) * 16; }
// BF16: 8 values per 16-byte core-matrix row, 4 chunks per 8-row group (SBO 512 B)
__host__ __device__ constexpr int tc_core_offset_bf(int r, int c) { return (r >> 3) * 512 + c * 128 + (r & 7) * 16; }

__host__ __device__ constexpr bool tc_split(int mode) { return mode == 1; }
__host__ __device__ constexpr int tc_mblock(int mode) { return mode == 2 ? kTcMBlockBf : kTcMBlock; }
__host__ __device__ constexpr int tc_btile(int mode) { return mode == 2 ? kTcBTileBf : kTcBTile; }

template <int kMode>
__host__ __device__ constexpr size_t tc_smem_bytes() {
    return 128 /* align */ + (tc_split(kMode) ? 2 : 1) * (tc_btile(kMode) + 2 * tc_mblock(kMode)) +
           tc_ring(tc_split(kMode)) * kTcPSlot * 4 + kTcXch * 4 + 32;
}

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t sbo = 768) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)(128 >> 4) << 16;                 // leading byte offset (K direction)
    d |= (uint64_t)(sbo >> 4) << 32;                 // stride byte offset (M/N direction)
    d |= (uint64_t)1 << 46;                          // descriptor version (sm_100)
    // base offset 0, lbo mode 0, layout type 0 = no swizzle
    return d;
}

// kind::tf32, D = F32, A = B = TF32, both K-major, N = 32, M = 128
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
// kind::f16, D = F32, A = B = BF16, both K-major, N = 32, M = 128
constexpr uint32_t kTcIdescBf = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Bounded wait for the phase of an mbarrier: false after about a second.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    const long long t0 = clock64();
    while (clock64() - t0 < kTcWaitCycles) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t ad, uint64_t bd, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "l"(ad), "l"(bd), "r"(kTcIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void tc_mma_bf16(uint32_t d, uint64_t ad, uint64_t bd, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "l"(ad), "l"(bd), "r"(kTcIdescBf), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
// two floats to a packed bf16x2 (round to nearest even); lo in the low half
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

template <class Epi, int kMode>
__global__ void __launch_bounds__(kTcThreads, kMode == 1 ? 3 : 4)
k_apply_tc(const __grid_constant__ TcKe ke, const Grid g, const float *__restrict__ p,
           const float *__restrict__ Eact, const int xchunk, const int ntz, Epi epi,
           const CGState *__restrict__ st, int *err) {
    if (blockIdx.z) {  // right-hand side of a batched solve
        const long long zr = blockIdx.z;
        p += zr * g.ndof;
        if (st) st += zr;
        epi.shift(zr, g.ndof);
    }
    if ((st && st->done) || epi.skip()) return;
    constexpr bool kSplit = tc_split(kMode), kBf = kMode == 2;
    constexpr int kMB = tc_mblock(kMode), kBT = tc_btile(kMode);
    extern __shared__ __align__(16) unsigned char tc_smem_raw[];
    const uint32_t raw_s = (uint32_t)__cvta_generic_to_shared(tc_smem_raw);
    unsigned char *base = tc_smem_raw + ((128 - (raw_s & 127)) & 127);
    unsigned char *Bh = base;
    unsigned char *Bl = Bh + kBT;                                // kSplit only
    unsigned char *Ah = base + (kSplit ? 2 : 1) * kBT;
    unsigned char *Al = Ah + 2 * kMB;                            // kSplit only
    float *ring = reinterpret_cast<float *>(Ah + (kSplit ? 2 : 1) * 2 * kMB);
    constexpr int R = tc_ring(kSplit);
    float *xch = ring + R * kTcPSlot;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(xch + kTcXch);  // two barriers
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 2);

    const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
    const int ty = blockIdx.x / ntz, tz = blockIdx.x % ntz;
    const int ey0 = ty * kTcNodesY - 1, ez0 = tz * kTcNodesZ - 1;
    const int ey = ey0 + w, ez = ez0 + l;
    const int ny = ey, nz = ez;  // node owned by this thread
    const bool owner = w >= 1 && l >= 1 && ny < g.nny && nz < g.nnz;
    const int x0 = blockIdx.y * xchunk;
    const int x1 = min(x0 + xchunk, g.nnx);
    const long long ncol = (long long)g.nny * g.nnz;
    const bool erow = ey >= 0 && ey < g.nely && ez >= 0 && ez < g.nelz;

    // ---- set-up: tensor memory, barriers, B operands --------------------------------
    if (w == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"((uint32_t)__cvta_generic_to_shared(tslot)), "r"(kTcCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(mbar)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(mbar + 1)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if constexpr (kBf) {
        for (int i = tid; i < 32 * 32; i += kTcThreads) reinterpret_cast<uint16_t *>(Bh)[i] = ke.bbf[i];
        // the zero K chunk (values 24..31) of every A row; the planes only rewrite chunks 0..2
        for (int r = tid; r < 256; r += kTcThreads)
            *reinterpret_cast<uint4 *>(Ah + (r >> 7) * kMB + tc_core_offset_bf(r & 127, 3)) = make_uint4(0u, 0u, 0u, 0u);
    } else {
        for (int i = tid; i < 32 * 24; i += kTcThreads) {
            reinterpret_cast<float *>(Bh)[i] = ke.bhi[i];
            if constexpr (kSplit) reinterpret_cast<float *>(Bl)[i] = ke.blo[i];
        }
    }
    // per-thread share of a staged node plane: offsets within a global node plane
    int loff[kTcLoads];
#pragma unroll
    for (int q = 0; q < kTcLoads; q++) {
        const int i = tid + q * kTcThreads;
        const int row = i / kTcPRow, rem = i - row * kTcPRow;
        const int y = ey0 + row, z = ez0 + rem / 3, c = rem % 3;
        const bool v = i < kTcPPlane && y >= 0 && y < g.nny && z >= 0 && z < g.nnz;
        loff[q] = v ? (y * g.nnz + z) * 3 + c : -1;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = *tslot;
    const uint32_t bar0 = (uint32_t)__cvta_generic_to_shared(mbar);
    const uint32_t ah_s = (uint32_t)__cvta_generic_to_shared(Ah);
    const uint32_t al_s = (uint32_t)__cvta_generic_to_shared(Al);
    const uint32_t bh_s = (uint32_t)__cvta_generic_to_shared(Bh);
    const uint32_t bl_s = (uint32_t)__cvta_generic_to_shared(Bl);

    auto slot_of = [&](int xk) { return ring + ((xk - x0 + 1) % R) * kTcPSlot; };
    auto load_plane = [&](int xk) {
        const bool pv = xk >= 0 && xk < g.nnx;
        const float *src = p + (pv ? (long long)xk * ncol * 3 : 0);
        float *dst = slot_of(xk);
#pragma unroll
        for (int q = 0; q < kTcLoads; q++) {
            const int i = tid + q * kTcThreads;
            if (i < kTcPPlane) {
                const bool v = pv && loff[q] >= 0;
                cp_async4(dst + i, v ? src + loff[q] : p, v);
            }
        }
    };
    auto load_e = [&](int k) {
        return (erow && k >= 0 && k < g.nelx) ? __ldg(Eact + ((long long)k * g.nely + ey) * g.nelz + ez) : 0.f;
    };

    float carry[3] = {0.f, 0.f, 0.f};
    float pc_cur[3] = {0.f, 0.f, 0.f}, pc_prev[3];
    double part[Epi::NV > 0 ? Epi::NV : 1];
#pragma unroll
    for (int k = 0; k < (Epi::NV > 0 ? Epi::NV : 1); k++) part[k] = 0.0;
    bool ok = true;
    uint32_t phbits = 0u;  // bit s: parity of the next phase of barrier s to wait for
    int pending = -1;  // stage of the last MMA whose completion nobody has waited for

    if (x0 < x1) {
        load_plane(x0 - 1);
        load_plane(x0);
        cp_async_commit();
#pragma unroll
        for (int j = 1; j <= R - 3; j++) {  // one commit group per plane from here on
            if (x0 + j <= x1) load_plane(x0 + j);
            cp_async_commit();
        }
        float e_next = load_e(x0 - 1);
        for (int k = x0 - 1; k <= x1; k++) {
            const bool build = k < x1;      // element plane k: A, MMA
            const bool epil = k >= x0;      // epilogue of element plane k-1
            // (a) node plane k+1 staged (planes k+2 .. k+R-2 may still be in flight); MMA(k-1)
            // done, so A and its TMEM stage may be reused
            cp_async_wait_pending<R - 3>();
            bool mine = ok;
            if (epil) mine = mine && mbar_wait(bar0 + 8u * ((k - 1) & 1), (phbits >> ((k - 1) & 1)) & 1u);
            ok = __syncthreads_and(mine);
            if (!ok) break;  // uniform: the tensor core did not finish in time
            if (epil) {
                phbits ^= 1u << ((k - 1) & 1);
                pending = -1;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // (b) prefetch node plane k+R-1 into the slot of plane k-1
            if (k + R - 1 <= x1) load_plane(k + R - 1);
            cp_async_commit();
            // (c) A(k): E_e u_e in the reference's local node order
            const float E = e_next;
#pragma unroll
            for (int c = 0; c < 3; c++) pc_prev[c] = pc_cur[c];
            if (build) {
                e_next = load_e(k + 1);
                const float *s0 = slot_of(k), *s1 = slot_of(k + 1);
                float u[24];
#pragma unroll
                for (int b = 0; b < 8; b++) {
                    const int bx = (b == 1 || b == 2 || b == 5 || b == 6);
                    const int by = (b == 2 || b == 3 || b == 6 || b == 7);
                    const int bz = (b >= 4);
                    const float *sb = (bx ? s1 : s0) + (w + by) * kTcPRow + (l + bz) * 3;
#pragma unroll
                    for (int c = 0; c < 3; c++) u[b * 3 + c] = sb[c];
                }
#pragma unroll
                for (int c = 0; c < 3; c++) pc_cur[c] = u[c];  // node (ey, ez) of plane k
                const int r = (w & 3) * 32 + l;
                unsigned char *ah = Ah + (w >> 2) * kMB;
                unsigned char *al = Al + (w >> 2) * kMB;
                if constexpr (kBf) {
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        uint32_t q[4];
#pragma unroll
                        for (int j = 0; j < 4; j++) q[j] = pack_bf16x2(E * u[8 * c + 2 * j], E * u[8 * c + 2 * j + 1]);
                        *reinterpret_cast<uint4 *>(ah + tc_core_offset_bf(r, c)) = make_uint4(q[0], q[1], q[2], q[3]);
                    }
                } else
#pragma unroll
                for (int c = 0; c < 6; c++) {
                    float hv[4], lv[4];
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const float a = E * u[4 * c + j];
                        hv[j] = to_tf32(a);
                        lv[j] = to_tf32(a - hv[j]);
                    }
                    *reinterpret_cast<float4 *>(ah + tc_core_offset(r, c)) = make_float4(hv[0], hv[1], hv[2], hv[3]);
                    if constexpr (kSplit)
                        *reinterpret_cast<float4 *>(al + tc_core_offset(r, c)) =
                            make_float4(lv[0], lv[1], lv[2], lv[3]);
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            // (d) MMA(k) into stage k%2
            if (build && tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t stage = (uint32_t)(k & 1);
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const uint32_t d = tbase + stage * 64u + (uint32_t)j * 32u;
                    if constexpr (kBf) {
#pragma unroll
                        for (int s = 0; s < 2; s++)  // K = 16 per MMA: values 0..15, 16..31
                            tc_mma_bf16(d, tc_desc(ah_s + j * kMB + s * 256, 512), tc_desc(bh_s + s * 256, 512), s > 0);
                    } else {
#pragma unroll
                        for (int s = 0; s < 3; s++) {
                            const uint64_t ad = tc_desc(ah_s + j * kMB + s * 256);
                            const uint64_t bd = tc_desc(bh_s + s * 256);
                            tc_mma(d, ad, bd, s > 0);
                            if constexpr (kSplit) {
                                tc_mma(d, ad, tc_desc(bl_s + s * 256), 1u);
                                tc_mma(d, tc_desc(al_s + j * kMB + s * 256), bd, 1u);
                            }
                        }
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             ::"r"(bar0 + 8u * stage) : "memory");
            }
            if (build) pending = k & 1;
            // (e) epilogue of element plane k-1 from stage (k-1)%2 (complete since (a))
            if (epil) {
                float y[32];
                {
                    const uint32_t taddr = tbase + ((uint32_t)((w & 3) * 32) << 16) + (uint32_t)(((k - 1) & 1) * 64) +
                                           (uint32_t)((w >> 2) * 32);
                    uint32_t rr[32];
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                        : "=r"(rr[0]), "=r"(rr[1]), "=r"(rr[2]), "=r"(rr[3]), "=r"(rr[4]), "=r"(rr[5]),
                          "=r"(rr[6]), "=r"(rr[7]), "=r"(rr[8]), "=r"(rr[9]), "=r"(rr[10]), "=r"(rr[11]),
                          "=r"(rr[12]), "=r"(rr[13]), "=r"(rr[14]), "=r"(rr[15]), "=r"(rr[16]), "=r"(rr[17]),
                          "=r"(rr[18]), "=r"(rr[19]), "=r"(rr[20]), "=r"(rr[21]), "=r"(rr[22]), "=r"(rr[23]),
                          "=r"(rr[24]), "=r"(rr[25]), "=r"(rr[26]), "=r"(rr[27]), "=r"(rr[28]), "=r"(rr[29]),
                          "=r"(rr[30]), "=r"(rr[31])
                        : "r"(taddr));
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int i = 0; i < 32; i++) y[i] = __uint_as_float(rr[i]);
                }
                // z-combine: node z gets this element's oz=0 corner and lane l-1's oz=1 corner
                float v[2][2][3];  // [ox][oy][c]
#pragma unroll
                for (int ox = 0; ox < 2; ox++)
#pragma unroll
                    for (int oy = 0; oy < 2; oy++)
#pragma unroll
                        for (int c = 0; c < 3; c++) {
                            const float up = __shfl_up_sync(0xffffffffu, y[3 * local_node(ox, oy, 1) + c], 1);
                            v[ox][oy][c] = y[3 * local_node(ox, oy, 0) + c] + (l > 0 ? up : 0.f);
                        }
                // y-combine: node row ey gets row ey's oy=0 part and row ey-1's oy=1 part
#pragma unroll
                for (int ox = 0; ox < 2; ox++)
#pragma unroll
                    for (int c = 0; c < 3; c++) xch[(ox * 3 + c) * kTcThreads + tid] = v[ox][1][c];
                __syncthreads();
                if (w >= 1) {
                    float tot[2][3];
#pragma unroll
                    for (int ox = 0; ox < 2; ox++)
#pragma unroll
                        for (int c = 0; c < 3; c++)
                            tot[ox][c] = v[ox][0][c] + xch[(ox * 3 + c) * kTcThreads + tid - 32];
                    if (owner && k - 1 >= x0) {
                        const long long dof0 = ((long long)(k - 1) * ncol + (long long)ny * g.nnz + nz) * 3;
                        float acc[3] = {carry[0] + tot[0][0], carry[1] + tot[0][1], carry[2] + tot[0][2]};
                        add_spring(g, dof0, acc, pc_prev);
                        epi.emit(dof0, acc, pc_prev, part);
                    }
#pragma unroll
                    for (int c = 0; c < 3; c++) carry[c] = tot[1][c];
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        }
        cp_async_wait_all();
    }

    if constexpr (Epi::NV > 0) {
        __shared__ double sh[32 * Epi::NV];
        double tot[Epi::NV];
        if (grid_sum<Epi::NV>(part, epi.partials, epi.counter, sh, tot)) {
            if (threadIdx.x == 0) epi.finalize(tot);
        }
    }
    if (!ok) {
        if (tid == 0 && err) atomicExch(err, 1);
        // give the last MMA one more bounded wait before the memory is released
        if (tid == 0 && pending >= 0) mbar_wait(bar0 + 8u * (uint32_t)pending, (phbits >> pending) & 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (w == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kTcCols));
    }
}

}  // namespace tpo
