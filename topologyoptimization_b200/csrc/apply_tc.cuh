// Tensor-core element contraction for the FP32 K*u of the mixed-precision solve.
//
// For every element plane the 24x24 product Y_e = Ke * u_e of 256 elements runs as two
// TF32 tcgen05.mma of shape M=128 (elements) x N=32 (24 outputs + 8 zero rows of Ke)
// x K=24 (u_e), A and B staged in shared memory in the canonical no-swizzle K-major
// core-matrix layout, the FP32 accumulator in tensor memory.  One thread per element
// reads its 24 outputs back with tcgen05.ld, scales them by E_e, and the node sums are
// formed with a warp shuffle along z (lanes are z-consecutive elements) and one shared-
// memory exchange along y (warps are y-consecutive element rows).  Nodes own their sum,
// as in k_apply: no atomics.
//
// CTA: 256 threads = 8 element rows x 32 elements; it owns the 7 x 31 nodes whose four
// (y,z)-adjacent elements all lie in the tile, and sweeps an x-chunk carrying the
// plane-k+1 partial sums, like k_apply.  Tiles overlap by one element row/column.
//
// Every mbarrier wait is bounded; on expiry the kernel records the failure in *err,
// stops issuing work, releases its tensor memory and returns.
#pragma once
#include "apply.cuh"

namespace tpo {

constexpr int kTcThreads = 256;
constexpr int kTcRowsE = 8;   // element rows per tile (y)
constexpr int kTcColsE = 32;  // elements per row (z)
constexpr int kTcNodesY = kTcRowsE - 1;
constexpr int kTcNodesZ = kTcColsE - 1;
constexpr int kTcPRow = (kTcColsE + 1) * 3;           // floats per staged node row
constexpr int kTcPPlane = (kTcRowsE + 1) * kTcPRow;   // floats per staged p plane
constexpr int kTcATile = 128 * 24 * 4;                // bytes per A tile (128 rows x 24 tf32)
constexpr int kTcBTile = 32 * 24 * 4;                 // bytes of the B tile (32 rows x 24 tf32)
constexpr int kTcXch = kTcThreads * 6;                // floats of the y-exchange buffer
constexpr long long kTcWaitCycles = 2000000000LL;  // about one second at B200 clocks

// Ke^T as the B operand: row n (output) = Ke row n for n < 24, zero rows 24..31;
// TF32-rounded on the host, already in core-matrix order (see tc_core_offset).
struct TcKe {
    float b[32 * 24];
};

// Byte offset of element (row r, k-chunk c of 4 values) in a K-major no-swizzle tile
// with 24 values per row: 8-row core matrices of 16-byte rows; the 6 chunks of one
// 8-row group are adjacent (LBO = 128 B) and groups are 768 B apart (SBO).
__host__ __device__ constexpr int tc_core_offset(int r, int c) { return (r >> 3) * 768 + c * 128 + (r & 7) * 16; }

__host__ __device__ constexpr size_t tc_smem_bytes() {
    return 1024 /* align */ + kTcBTile + 2 * kTcATile + 2 * kTcPPlane * 4 + kTcXch * 4 + 64;
}

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)(128 >> 4) << 16;                 // leading byte offset (K direction)
    d |= (uint64_t)(768 >> 4) << 32;                 // stride byte offset (M/N direction)
    d |= (uint64_t)1 << 46;                          // descriptor version (sm_100)
    // base offset 0, lbo mode 0, layout type 0 = no swizzle
    return d;
}

// kind::tf32, D = F32, A = B = TF32, both K-major, N = 32, M = 128
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

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

template <class Epi>
__global__ void __launch_bounds__(kTcThreads, 3)
k_apply_tc(const __grid_constant__ TcKe ke, const Grid g, const float *__restrict__ p,
           const float *__restrict__ Eact, const int xchunk, const int ntz, Epi epi,
           const CGState *__restrict__ st, int *err) {
    if ((st && st->done) || epi.skip()) return;
    extern __shared__ __align__(16) unsigned char tc_smem_raw[];
    // 1024-byte aligned base for the operand tiles
    const uint32_t raw_s = (uint32_t)__cvta_generic_to_shared(tc_smem_raw);
    const uint32_t pad = (1024 - (raw_s & 1023)) & 1023;
    unsigned char *base = tc_smem_raw + pad;
    unsigned char *Bs = base;
    unsigned char *As = Bs + kTcBTile;
    float *pbuf = reinterpret_cast<float *>(As + 2 * kTcATile);
    float *xch = pbuf + 2 * kTcPPlane;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(xch + kTcXch);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);

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

    // ---- set-up: tensor memory, barrier, B operand ---------------------------------
    if (w == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"((uint32_t)__cvta_generic_to_shared(tslot)), "r"(64u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < 32 * 24; i += kTcThreads) reinterpret_cast<float *>(Bs)[i] = ke.b[i];
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = *tslot;
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(mbar);
    const uint32_t a_s = (uint32_t)__cvta_generic_to_shared(As);
    const uint32_t b_s = (uint32_t)__cvta_generic_to_shared(Bs);

    auto load_plane = [&](int xk, float *buf) {
        const bool pv = xk >= 0 && xk < g.nnx;
        for (int i = tid; i < kTcPPlane; i += kTcThreads) {
            const int row = i / kTcPRow, rem = i - row * kTcPRow;
            const int y = ey0 + row, z = ez0 + rem / 3, c = rem % 3;
            const bool v = pv && y >= 0 && y < g.nny && z >= 0 && z < g.nnz;
            const float *src = v ? p + (((long long)xk * g.nny + y) * g.nnz + z) * 3 + c : p;
            cp_async4(buf + i, src, v);
        }
    };
    // my four nodes (ey+by, ez+bz) of a staged plane: q[by][bz][c]
    auto read_nodes = [&](const float *buf, float (&q)[2][2][3]) {
#pragma unroll
        for (int by = 0; by < 2; by++)
#pragma unroll
            for (int bz = 0; bz < 2; bz++)
#pragma unroll
                for (int c = 0; c < 3; c++) q[by][bz][c] = buf[(w + by) * kTcPRow + (l + bz) * 3 + c];
    };

    float Q0[2][2][3], Q1[2][2][3];
    float carry[3] = {0.f, 0.f, 0.f};
    double part[Epi::NV > 0 ? Epi::NV : 1];
#pragma unroll
    for (int k = 0; k < (Epi::NV > 0 ? Epi::NV : 1); k++) part[k] = 0.0;
    bool ok = true;
    uint32_t phase = 0;

    if (x0 < x1) {
        load_plane(x0 - 1, pbuf);
        load_plane(x0, pbuf + kTcPPlane);
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        read_nodes(pbuf, Q0);
        int slot = 0;
        for (int k = x0 - 1; k < x1; k++) {
            read_nodes(pbuf + (slot ^ 1) * kTcPPlane, Q1);
            const float E = (erow && k >= 0 && k < g.nelx) ? Eact[((long long)k * g.nely + ey) * g.nelz + ez] : 0.f;
            __syncthreads();  // slot (plane k) consumed by everyone
            if (k + 1 < x1) load_plane(k + 2, pbuf + slot * kTcPPlane);
            cp_async_commit();

            // A row of this element: u_e in the reference's local order, TF32-rounded
            {
                float u[24];
#pragma unroll
                for (int b = 0; b < 8; b++) {
                    const int bx = (b == 1 || b == 2 || b == 5 || b == 6);
                    const int by = (b == 2 || b == 3 || b == 6 || b == 7);
                    const int bz = (b >= 4);
#pragma unroll
                    for (int c = 0; c < 3; c++) u[b * 3 + c] = to_tf32(bx ? Q1[by][bz][c] : Q0[by][bz][c]);
                }
                unsigned char *at = As + (w >> 2) * kTcATile;
                const int r = (w & 3) * 32 + l;
#pragma unroll
                for (int c = 0; c < 6; c++)
                    *reinterpret_cast<float4 *>(at + tc_core_offset(r, c)) =
                        make_float4(u[4 * c], u[4 * c + 1], u[4 * c + 2], u[4 * c + 3]);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0 && ok) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
                for (int j = 0; j < 2; j++) {
#pragma unroll
                    for (int s = 0; s < 3; s++) {
                        const uint64_t ad = tc_desc(a_s + j * kTcATile + s * 256);
                        const uint64_t bd = tc_desc(b_s + s * 256);
                        const uint32_t acc = s > 0;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                            ::"r"(tbase + j * 32), "l"(ad), "l"(bd), "r"(kTcIdesc), "r"(acc),
                            "r"(0u), "r"(0u), "r"(0u), "r"(0u));
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             ::"r"(bar) : "memory");
            }
            ok = __syncthreads_and(ok && mbar_wait(bar, phase));
            if (!ok) {  // uniform: the tensor core did not finish in time
                if (tid == 0 && err) atomicExch(err, 1);
                break;
            }
            phase ^= 1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float y[32];
            {
                const uint32_t taddr = tbase + ((uint32_t)((w & 3) * 32) << 16) + (uint32_t)((w >> 2) * 32);
                uint32_t rr[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                    "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(rr[0]), "=r"(rr[1]), "=r"(rr[2]), "=r"(rr[3]), "=r"(rr[4]), "=r"(rr[5]), "=r"(rr[6]),
                      "=r"(rr[7]), "=r"(rr[8]), "=r"(rr[9]), "=r"(rr[10]), "=r"(rr[11]), "=r"(rr[12]),
                      "=r"(rr[13]), "=r"(rr[14]), "=r"(rr[15]), "=r"(rr[16]), "=r"(rr[17]), "=r"(rr[18]),
                      "=r"(rr[19]), "=r"(rr[20]), "=r"(rr[21]), "=r"(rr[22]), "=r"(rr[23]), "=r"(rr[24]),
                      "=r"(rr[25]), "=r"(rr[26]), "=r"(rr[27]), "=r"(rr[28]), "=r"(rr[29]), "=r"(rr[30]),
                      "=r"(rr[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int i = 0; i < 32; i++) y[i] = E != 0.f ? __uint_as_float(rr[i]) * E : 0.f;
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
                    for (int c = 0; c < 3; c++) tot[ox][c] = v[ox][0][c] + xch[(ox * 3 + c) * kTcThreads + tid - 32];
                if (owner && k >= x0) {
                    const long long dof0 = ((long long)k * ncol + (long long)ny * g.nnz + nz) * 3;
                    const float acc[3] = {carry[0] + tot[0][0], carry[1] + tot[0][1], carry[2] + tot[0][2]};
                    const float pc[3] = {Q0[0][0][0], Q0[0][0][1], Q0[0][0][2]};
                    epi.emit(dof0, acc, pc, part);
                }
#pragma unroll
                for (int c = 0; c < 3; c++) carry[c] = tot[1][c];
            }
#pragma unroll
            for (int by = 0; by < 2; by++)
#pragma unroll
                for (int bz = 0; bz < 2; bz++)
#pragma unroll
                    for (int c = 0; c < 3; c++) Q0[by][bz][c] = Q1[by][bz][c];
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            cp_async_wait_all();
            __syncthreads();  // TMEM reads, the exchange buffer and the A tiles are free again
            slot ^= 1;
        }
    }

    if constexpr (Epi::NV > 0) {
        __shared__ double sh[32 * Epi::NV];
        double tot[Epi::NV];
        if (grid_sum<Epi::NV>(part, epi.partials, epi.counter, sh, tot)) {
            if (threadIdx.x == 0) epi.finalize(tot);
        }
    }
    if (!ok) {
        // give the outstanding MMAs one more bounded wait before the memory is released
        cp_async_wait_all();
        if (tid == 0) mbar_wait(bar, phase);
    }
    __syncthreads();
    if (w == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(64u));
    }
}

}  // namespace tpo
