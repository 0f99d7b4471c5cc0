// Host side of libtpo: problem handles, multigrid hierarchy, PCG drivers, SIMP step and
// the C ABI declared in include/tpo.h.  Every exported function catches all errors and
// returns a tpo_status.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <type_traits>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tpo.h"
#include "apply.cuh"
#include "apply_tc.cuh"
#include "apply_walsh.cuh"
#include "kernels.cuh"
#include "mg_kernels.cuh"

using namespace tpo;

namespace {

thread_local std::string g_err;

struct Failure {
    tpo_status st;
    std::string msg;
};

[[noreturn]] void fail(tpo_status s, const std::string &m) { throw Failure{s, m}; }

#define CK(call)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) {                                                                    \
            if (e_ == cudaErrorMemoryAllocation) {                                                  \
                cudaGetLastError();                                                                 \
                fail(TPO_OOM, std::string(#call) + ": " + cudaGetErrorString(e_));                  \
            }                                                                                       \
            fail(TPO_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_) + " at " +      \
                                     std::to_string(__LINE__));                                     \
        }                                                                                           \
    } while (0)
// Every kernel launch of the library is followed by CKL(), which also counts it.
std::atomic<long long> g_launches{0};
#define CKL()                         \
    do {                              \
        CK(cudaGetLastError());       \
        g_launches.fetch_add(1);      \
    } while (0)

template <typename F>
tpo_status guard(F &&f) {
    try {
        f();
        g_err.clear();
        return TPO_OK;
    } catch (const Failure &e) {
        g_err = e.msg;
        return e.st;
    } catch (const std::bad_alloc &) {
        g_err = "host allocation failed";
        return TPO_OOM;
    } catch (const std::exception &e) {
        g_err = e.what();
        return TPO_CUDA_ERROR;
    }
}

template <typename T>
T *dalloc(size_t n) {
    void *p = nullptr;
    if (n == 0) n = 1;
    CK(cudaMalloc(&p, n * sizeof(T)));
    return static_cast<T *>(p);
}
template <typename T>
void dfree(T *&p) {
    if (p) cudaFree(p);
    p = nullptr;
}

int g_num_sms = 0;

void check_device() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        fail(TPO_NO_DEVICE, "no CUDA device");
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, dev));
    if (prop.major < 10) fail(TPO_NO_DEVICE, "libtpo is built for sm_100a; device is sm_" +
                                                 std::to_string(prop.major) + std::to_string(prop.minor));
    g_num_sms = prop.multiProcessorCount;
}

inline unsigned nblk(long long n, int t = 256) { return (unsigned)std::max(1LL, (n + t - 1) / t); }
inline unsigned red_blocks() { return (unsigned)std::max(1, (g_num_sms ? g_num_sms : 148) * 4); }

KeParam<double> make_ke(const double *Ke) {
    KeParam<double> k;
    std::memcpy(k.v, Ke, sizeof k.v);
    return k;
}
KeParam<float> make_kef(const double *Ke) {
    KeParam<float> k;
    for (int i = 0; i < 576; i++) k.v[i] = (float)Ke[i];
    return k;
}
// Walsh-block constants of a hex8 element matrix (apply_walsh.cuh): B = W^T Ke W / 64 in
// the basis w_(sigma,c)[b, c'] = delta(c, c') (-1)^(sigma . b) over the corners b of the
// reference's local order.  False when B is not the block pattern of a cube element (a
// matrix without the cube's symmetries).  `general` is set when the rigid-body relations
// of lk(nu) (p = q, s = 0) fail beyond double rounding, as they do for a Ke rounded to
// single precision (the Float32Array KEflat of gpu-fea-solver.js); FP64 applies then use
// the general blocks, which reproduce that Ke exactly, and FP32 applies (preconditioner
// and inner solves) the nearest lk-form blocks, p = q = (p + q) / 2 and s = 0.
namespace walsh {
constexpr int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
struct Id {
    int sx, sy, sz, c;
};
constexpr int idx(Id i) { return (i.sx + 2 * i.sy + 4 * i.sz) * 3 + i.c; }
}  // namespace walsh

template <typename T>
bool make_walsh_ke(const double *Ke, WalshKe<T> &out) {
    using walsh::Id;
    using walsh::idx;
    double W[24][24];  // W[3b + c][idx(sigma, c')]
    for (int b = 0; b < 8; b++)
        for (int c = 0; c < 3; c++)
            for (int sg = 0; sg < 8; sg++)
                for (int c2 = 0; c2 < 3; c2++) {
                    const int e = (sg & 1) * walsh::kCorner[b][0] + ((sg >> 1) & 1) * walsh::kCorner[b][1] +
                                  ((sg >> 2) & 1) * walsh::kCorner[b][2];
                    W[3 * b + c][sg * 3 + c2] = c == c2 ? ((e & 1) ? -1.0 : 1.0) : 0.0;
                }
    double KW[24][24], B[24][24], mx = 0.0;
    for (int i = 0; i < 24; i++)
        for (int j = 0; j < 24; j++) {
            double acc = 0.0;
            for (int k = 0; k < 24; k++) acc += Ke[i * 24 + k] * W[k][j];
            KW[i][j] = acc;
            mx = std::max(mx, std::fabs(Ke[i * 24 + j]));
        }
    for (int i = 0; i < 24; i++)
        for (int j = 0; j < 24; j++) {
            double acc = 0.0;
            for (int k = 0; k < 24; k++) acc += W[k][i] * KW[k][j];
            B[i][j] = acc / 64.0;
        }
    const double a = B[idx({1, 1, 0, 2})][idx({1, 1, 0, 2})], b = B[idx({1, 1, 0, 2})][idx({1, 0, 1, 1})];
    const double p = B[idx({1, 0, 0, 1})][idx({1, 0, 0, 1})], q = B[idx({1, 0, 0, 1})][idx({0, 1, 0, 0})];
    const double d = B[idx({1, 1, 1, 2})][idx({1, 1, 1, 2})], s = B[idx({0, 0, 0, 0})][idx({0, 0, 0, 0})];
    const double e = B[idx({1, 1, 0, 1})][idx({1, 1, 0, 1})], f = B[idx({1, 1, 0, 1})][idx({1, 0, 1, 2})];
    const double g = B[idx({1, 0, 0, 0})][idx({1, 0, 0, 0})], h = B[idx({1, 0, 0, 0})][idx({0, 1, 0, 1})];
    double M[24][24] = {};
    auto block = [&](std::initializer_list<Id> ids, double dg, double od) {
        for (Id i : ids)
            for (Id j : ids) M[idx(i)][idx(j)] = idx(i) == idx(j) ? dg : od;
    };
    block({{1, 1, 0, 2}, {1, 0, 1, 1}, {0, 1, 1, 0}}, a, b);  // twist
    block({{1, 0, 0, 0}, {0, 1, 0, 1}, {0, 0, 1, 2}}, g, h);  // normal strains
    block({{1, 0, 0, 1}, {0, 1, 0, 0}}, p, q);                // shear xy
    block({{1, 0, 0, 2}, {0, 0, 1, 0}}, p, q);                // shear xz
    block({{0, 1, 0, 2}, {0, 0, 1, 1}}, p, q);                // shear yz
    block({{1, 1, 1, 2}}, d, d);
    block({{1, 1, 1, 1}}, d, d);
    block({{1, 1, 1, 0}}, d, d);
    block({{1, 1, 0, 1}, {1, 0, 1, 2}}, e, f);  // bending about x
    block({{1, 1, 0, 0}, {0, 1, 1, 2}}, e, f);  // bending about y
    block({{1, 0, 1, 0}, {0, 1, 1, 1}}, e, f);  // bending about z
    block({{0, 0, 0, 0}}, s, s);                // rigid translations
    block({{0, 0, 0, 1}}, s, s);
    block({{0, 0, 0, 2}}, s, s);
    for (int i = 0; i < 24; i++)
        for (int j = 0; j < 24; j++)
            if (!(std::fabs(B[i][j] - M[i][j]) <= 1e-12 * mx)) return false;  // NaN fails too
    const bool general = std::fabs(p - q) > 1e-13 * mx || std::fabs(s) > 1e-13 * mx;
    const bool exact_form = std::is_same_v<T, float> || !general;
    out.a1 = (T)(a - b);
    out.a2 = (T)b;
    out.p = (T)(exact_form ? 0.5 * (p + q) : p);
    out.q = (T)(exact_form ? 0.5 * (p + q) : q);
    out.s = (T)(exact_form ? 0.0 : s);
    out.general = exact_form ? 0 : 1;
    out.d = (T)d;
    out.e = (T)e;
    out.f = (T)f;
    out.g1 = (T)(g - h);
    out.g2 = (T)h;
    return true;
}

void device_lk(double nu, double *Ke_host) {
    double *d = dalloc<double>(576);
    k_lk<<<1, 576>>>(nu, d);
    CKL();
    CK(cudaMemcpy(Ke_host, d, 576 * sizeof(double), cudaMemcpyDeviceToHost));
    dfree(d);
}

// ---- apply launch ---------------------------------------------------------------------
struct ApplyShape {
    dim3 grid;
    int xchunk;
    size_t smem;
};

// Grid of the apply kernel: ceil(ncol / TOUT) column tiles times nch x-chunks.  Every
// chunk recomputes one element plane, and the launch runs in waves of `conc` resident
// CTAs, so the chunk count minimises waves * (planes per chunk + 1).
// Valid x-chunk counts of a grid (every chunk non-empty), ordered by that cost.
template <typename T>
std::vector<int> apply_chunk_candidates(const Grid &g, int conc) {
    if (walsh_out_cols<T>(g.nnz) <= 0) return {};
    const long long ncol = (long long)g.nny * g.nnz;
    const long long colb = (ncol + walsh_out_cols<T>(g.nnz) - 1) / walsh_out_cols<T>(g.nnz);
    std::vector<std::pair<long long, int>> c;
    for (int nch = 1; nch <= std::min(g.nnx, 512); nch++) {
        const int xch = (g.nnx + nch - 1) / nch;
        if ((g.nnx + xch - 1) / xch != nch) continue;
        c.push_back({((colb * nch + conc - 1) / conc) * (xch + 1), nch});
    }
    std::stable_sort(c.begin(), c.end());
    std::vector<int> out;
    for (auto &v : c) out.push_back(v.second);
    return out;
}

template <typename T>
ApplyShape apply_shape(const Grid &g, int conc, bool tuned = false) {
    ApplyShape s;
    const long long ncol = (long long)g.nny * g.nnz;
    const int tout = walsh_out_cols<T>(g.nnz);
    if (tout <= 0)
        fail(TPO_BAD_ARG, "grid too deep in z for the apply kernel's tiles (nelz + 2 must be below " +
                              std::to_string(WTile<T>::NEB) + ")");
    const long long colb = (ncol + tout - 1) / tout;
    conc = std::max(conc, 1);
    long long best = -1;
    int best_nch = 1;
    const int max_nch = std::min(g.nnx, 512);
    for (int nch = 1; nch <= max_nch; nch++) {
        const int xch = (g.nnx + nch - 1) / nch;
        const int n2 = (g.nnx + xch - 1) / xch;
        if (n2 != nch) continue;
        const long long waves = (colb * n2 + conc - 1) / conc;
        const long long cost = waves * (xch + 1);
        if (best < 0 || cost < best) {
            best = cost;
            best_nch = nch;
        }
    }
    const int tn = g.nch[sizeof(T) == 8 ? 1 : 0];
    if (tuned && tn > 0 && tn <= g.nnx) best_nch = tn;
    s.xchunk = (g.nnx + best_nch - 1) / best_nch;
    s.grid = dim3((unsigned)colb, (unsigned)((g.nnx + s.xchunk - 1) / s.xchunk), 1);
    s.smem = walsh_smem_bytes<T>(g);
    return s;
}

template <typename T, class Epi>
size_t &apply_configured() {
    static size_t configured = 48 * 1024;
    return configured;
}
// Resident CTAs of one k_apply_w instantiation across the device, at its configured
// (largest) shared-memory size.
template <typename T, class Epi>
int &apply_conc() {
    static int conc = 0;
    return conc;
}
// Resident CTAs per SM of the apply kernel from its resources: shared memory (with the
// 1 KB the runtime reserves per CTA), registers and threads.
template <typename T, class Epi, bool kGen>
int apply_per_sm(size_t smem) {
    cudaFuncAttributes fa{};
    CK(cudaFuncGetAttributes(&fa, k_apply_w<T, Epi, kGen>));
    int dev = 0, smem_sm = 0, regs_sm = 0, thr_sm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    CK(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev));
    CK(cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev));
    const size_t per_cta = smem + fa.sharedSizeBytes + 1024;
    const int by_smem = (int)(smem_sm / std::max(per_cta, (size_t)1));
    const int regs = std::max(fa.numRegs, 1) * WTile<T>::NT;
    const int by_regs = regs_sm / regs;
    const int by_thr = thr_sm / WTile<T>::NT;
    return std::max(1, std::min(by_smem, std::min(by_regs, by_thr)));
}
// Raise the dynamic shared-memory limit of one k_apply_w instantiation and record its
// occupancy.  Called when a problem is created (never during stream capture).
// (FP64 instantiations come in both forms of the Walsh blocks; FP32 only in lk's.)
template <typename T, class Epi>
void configure_apply(size_t smem) {
    constexpr bool kDouble = std::is_same_v<T, double>;
    if (smem > apply_configured<T, Epi>()) {
        CK(cudaFuncSetAttribute(k_apply_w<T, Epi, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        if constexpr (kDouble)
            CK(cudaFuncSetAttribute(k_apply_w<T, Epi, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        apply_configured<T, Epi>() = smem;
    }
    int per_sm = apply_per_sm<T, Epi, false>(smem);
    if constexpr (kDouble) per_sm = std::min(per_sm, apply_per_sm<T, Epi, true>(smem));
    const int conc = per_sm * (g_num_sms ? g_num_sms : 148);
    if (apply_conc<T, Epi>() == 0 || conc < apply_conc<T, Epi>()) apply_conc<T, Epi>() = conc;
}

template <typename T, class Epi>
void launch_apply(cudaStream_t st, const Grid &g, const WalshKe<T> &wk, const T *p, const T *Eact, const Epi &epi,
                  const CGState *cg, int nrhs = 1) {
    // the measured shape for launches without a grid-wide reduction (a reduction's order
    // follows the block count, which stays the cost model's so that results do not depend
    // on timing); batched launches keep the model, which counts their extra CTAs
    const ApplyShape s = apply_shape<T>(g, apply_conc<T, Epi>(), Epi::NV == 0 && nrhs == 1);
    if (s.smem > apply_configured<T, Epi>()) fail(TPO_BAD_ARG, "apply shared memory was not configured");
    const dim3 grid(s.grid.x, s.grid.y, (unsigned)nrhs);
    if constexpr (std::is_same_v<T, double>) {
        if (wk.general) {
            k_apply_w<T, Epi, true><<<grid, WTile<T>::NT, s.smem, st>>>(wk, g, p, Eact, s.xchunk, epi, cg);
            CKL();
            return;
        }
    }
    k_apply_w<T, Epi, false><<<grid, WTile<T>::NT, s.smem, st>>>(wk, g, p, Eact, s.xchunk, epi, cg);
    CKL();
}

void configure_all_applies(const Grid *levels, int nl) {
    size_t md = 0, mf = 0;
    for (int i = 0; i < nl; i++) {
        if (walsh_out_cols<double>(levels[i].nnz) <= 0)
            fail(TPO_BAD_ARG, "grid too deep in z for the apply kernel's tiles (nelz + 2 must be below " +
                                  std::to_string(WTile<double>::NEB) + ")");
        md = std::max(md, walsh_smem_bytes<double>(levels[i]));
        mf = std::max(mf, walsh_smem_bytes<float>(levels[i]));
    }
    if (md > 227 * 1024 || mf > 227 * 1024) fail(TPO_BAD_ARG, "grid too deep in z for the apply kernel's tiles");
    configure_apply<double, EpiStore<double>>(md);
    configure_apply<double, EpiSmooth<double>>(md);
    configure_apply<double, EpiResidual<double>>(md);
    configure_apply<double, EpiCG<double>>(md);
    configure_apply<double, EpiDefect>(md);
    configure_apply<double, EpiSmoothDot<double>>(md);
    configure_apply<double, EpiCheb<double>>(md);
    configure_apply<double, EpiBddcCoarse<double>>(md);
    configure_apply<float, EpiCheb<float>>(mf);
    configure_apply<float, EpiStore<float>>(mf);
    configure_apply<float, EpiSmooth<float>>(mf);
    configure_apply<float, EpiResidual<float>>(mf);
    configure_apply<float, EpiCG<float>>(mf);
}

// ---- tensor-core apply ------------------------------------------------------------------
// Ke^T as the TF32 B operand in the kernel's core-matrix order (rows 24..31 zero), each
// value rounded to TF32 (nearest, ties away from zero), as cvt.rna.tf32.f32 does.
namespace tf32h {
// cvt.rna.tf32.f32 on the host: round to nearest, ties away from zero, 10 mantissa bits
float rna(float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    u = (u + 0x1000u) & 0xFFFFE000u;
    std::memcpy(&v, &u, 4);
    return v;
}
// float -> bf16 bits, round to nearest, ties to even (as cvt.rn.bf16x2.f32), finite inputs
uint16_t bf16_rne(float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
}  // namespace tf32h

// Ke^T as the TF32 B operands in the kernel's core-matrix order (rows 24..31 zero):
// high part rna(Ke) and low part rna(Ke - high).
TcKe make_tc_ke(const double *Ke) {
    TcKe t;
    std::memset(&t, 0, sizeof t);
    for (int n = 0; n < 24; n++)
        for (int k = 0; k < 24; k++) {
            const float v = (float)Ke[n * 24 + k];
            const float hi = tf32h::rna(v);
            const int o = tc_core_offset(n, k / 4) / 4 + (k % 4);
            t.bhi[o] = hi;
            t.blo[o] = tf32h::rna(v - hi);
            t.bbf[tc_core_offset_bf(n, k / 8) / 2 + (k % 8)] = tf32h::bf16_rne(v);
        }
    return t;
}

template <class Epi, int kMode>
int &tc_conc() {
    static int conc = 0;
    return conc;
}
template <class Epi, int kMode>
void configure_tc() {
    if (tc_conc<Epi, kMode>()) return;
    CK(cudaFuncSetAttribute(k_apply_tc<Epi, kMode>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)tc_smem_bytes<kMode>()));
    // Resident CTAs per SM from the kernel's registers, shared memory, threads and tensor
    // memory (512 columns per SM).  cudaOccupancyMaxActiveBlocksPerMultiprocessor reports
    // 1 for these tcgen05 kernels, below what the SM runs (4 on B200 for the TF32 variant).
    cudaFuncAttributes fa{};
    CK(cudaFuncGetAttributes(&fa, k_apply_tc<Epi, kMode>));
    int dev = 0, regs_sm = 0, smem_sm = 0, smem_rsv = 0, thr_sm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev));
    CK(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    CK(cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    CK(cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev));
    const int regs_warp = ((std::max(fa.numRegs, 1) * 32 + 255) / 256) * 256;  // per-warp allocation unit
    const int by_regs = regs_sm / (regs_warp * (kTcThreads / 32));
    const int by_smem = smem_sm / (int)(tc_smem_bytes<kMode>() + fa.sharedSizeBytes + smem_rsv);
    const int by_thr = thr_sm / kTcThreads;
    const int by_tmem = 512 / (int)kTcCols;
    const int per_sm = std::max(1, std::min(std::min(by_regs, by_smem), std::min(by_thr, by_tmem)));
    tc_conc<Epi, kMode>() = per_sm * (g_num_sms ? g_num_sms : 148);
}
template <int kMode>
void configure_tc_all() {
    configure_tc<EpiStore<float>, kMode>();
    configure_tc<EpiSmooth<float>, kMode>();
    configure_tc<EpiResidual<float>, kMode>();
    configure_tc<EpiCG<float>, kMode>();
    configure_tc<EpiCheb<float>, kMode>();
}
void configure_all_tc() {
    configure_tc_all<0>();
    configure_tc_all<1>();
    configure_tc_all<2>();
}

template <class Epi, int kMode>
void launch_apply_tc_t(cudaStream_t st, const Grid &g, const TcKe &tke, const float *p, const float *Eact,
                       const Epi &epi, const CGState *cg, int *err, int nrhs) {
    if ((long long)g.nny * g.nnz * 3 >= (1LL << 31)) fail(TPO_BAD_ARG, "node plane too large for the tensor-core apply");
    const int nty = (g.nny + kTcNodesY - 1) / kTcNodesY, ntz = (g.nnz + kTcNodesZ - 1) / kTcNodesZ;
    const long long tiles = (long long)nty * ntz;
    const int conc = std::max(1, tc_conc<Epi, kMode>());
    long long best = -1;
    int best_nch = 1;
    for (int nch = 1; nch <= std::min(g.nnx, 512); nch++) {
        const int xch = (g.nnx + nch - 1) / nch;
        if ((g.nnx + xch - 1) / xch != nch) continue;
        const long long cost = ((tiles * nch + conc - 1) / conc) * (xch + 2);
        if (best < 0 || cost < best) {
            best = cost;
            best_nch = nch;
        }
    }
    const int xchunk = (g.nnx + best_nch - 1) / best_nch;
    k_apply_tc<Epi, kMode><<<dim3((unsigned)tiles, (unsigned)best_nch, (unsigned)nrhs), kTcThreads,
                             tc_smem_bytes<kMode>(), st>>>(
        tke, g, p, Eact, xchunk, ntz, epi, cg, err);
    CKL();
}
template <class Epi>
void launch_apply_tc(cudaStream_t st, const Grid &g, const TcKe &tke, const float *p, const float *Eact,
                     const Epi &epi, const CGState *cg, int *err, int mode, int nrhs = 1) {
    if (mode == 1) launch_apply_tc_t<Epi, 1>(st, g, tke, p, Eact, epi, cg, err, nrhs);
    else if (mode == 2) launch_apply_tc_t<Epi, 2>(st, g, tke, p, Eact, epi, cg, err, nrhs);
    else launch_apply_tc_t<Epi, 0>(st, g, tke, p, Eact, epi, cg, err, nrhs);
}

// ---- host-side hierarchy bookkeeping ------------------------------------------------
// _downsampleFixedMaskBy2 (js/optimizer-worker-3d.js:384-406): injection from fine node
// min(2c, nF-1).
std::vector<uint8_t> downsample_fixed(const std::vector<uint8_t> &ff, const Grid &gf, const Grid &gc) {
    std::vector<uint8_t> fc((size_t)gc.ndof, 0);
    for (int cz = 0; cz < gc.nnz; cz++) {
        const int fz = std::min(2 * cz, gf.nnz - 1);
        for (int cy = 0; cy < gc.nny; cy++) {
            const int fy = std::min(2 * cy, gf.nny - 1);
            for (int cx = 0; cx < gc.nnx; cx++) {
                const int fx = std::min(2 * cx, gf.nnx - 1);
                const long long nF = ((long long)fx * gf.nny + fy) * gf.nnz + fz;
                const long long nC = ((long long)cx * gc.nny + cy) * gc.nnz + cz;
                for (int d = 0; d < 3; d++) fc[3 * nC + d] = ff[3 * nF + d];
            }
        }
    }
    return fc;
}

// Captured PCG iteration variants (enqueue_iteration's mode).
// Modes of the captured PCG iteration (enqueue_iteration); kModeStride more: the same
// iteration over a batch of right-hand sides.
constexpr int kModeStride = 12;
constexpr int kModeBddc = 10;
constexpr int kModeF32Bf16 = 11;  // FP64 PCG, FP32 V-cycle with BF16 tensor-core fine-level applies
constexpr int kIterModes = 2 * kModeStride;

struct Level {
    Grid g{};
    bool dense = false;
    uint8_t *fixed = nullptr;
    double *E = nullptr, *Eact = nullptr, *invD = nullptr;
    float *Eact32 = nullptr, *invD32 = nullptr;
    double *b = nullptr, *x = nullptr, *xt = nullptr, *res = nullptr;
    float *b32 = nullptr, *x32 = nullptr, *xt32 = nullptr, *res32 = nullptr;
    double *K = nullptr;
    double *Kinv = nullptr, *Lw = nullptr, *Yw = nullptr;  // coarsest level, direct solve
    cudaGraphExec_t gj = nullptr;                           // its n Gauss-Jordan sweeps as one graph
    double omega = 0.5;         // Jacobi damping of this level (host value, fixed at creation)
    // Chebyshev smoothing (structured levels, chebyshev option): sweep 0 is damped Jacobi
    // with 1 / theta, sweep k >= 1 uses (cheb_cd[k], cheb_cr[k]); one coefficient pair per
    // sweep of the longest sequence a V-cycle runs on the level (nu1, nu2, or nu1 +
    // coarse_iters on a structured coarsest level)
    int cheb = 0;
    double cheb_w0 = 0.0;
    std::vector<double> cheb_cd, cheb_cr;
    double *womega = nullptr;   // dense levels under safe_omega: damping set on the device
};

}  // namespace

// Buffers of a batched solve: nb right-hand sides, each vector nb x ndof (RHS-major), one
// CGState, compliance and dot counter per right-hand side, and per-level V-cycle buffers.
struct tpo_batch {
    int nb = 0;
    bool f32 = false;
    double *U = nullptr, *F = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr;
    float *r32 = nullptr, *z32 = nullptr;
    CGState *st = nullptr, *st_host = nullptr;
    double *partials = nullptr, *scal = nullptr, *scal_host = nullptr;
    unsigned *dot_counter = nullptr;
    double *Lb[kMaxLevels] = {}, *Lx[kMaxLevels] = {}, *Lxt[kMaxLevels] = {}, *Lres[kMaxLevels] = {};
    float *Lb32[kMaxLevels] = {}, *Lx32[kMaxLevels] = {}, *Lxt32[kMaxLevels] = {}, *Lres32[kMaxLevels] = {};
};

struct tpo_problem {
    Grid g{};
    int nl = 0;
    Level L[kMaxLevels];
    tpo_mg_opts mg{};
    double Ke[576];
    KeParam<double> ke;   // full matrix: diagonal, energy, Galerkin kernels
    KeParam<float> kef;
    WalshKe<double> wk;   // Walsh-block constants: structured apply kernels
    WalshKe<float> wkf;
    cudaStream_t s = nullptr;    // stream all work of the problem runs on
    cudaStream_t own = nullptr;  // the library-created stream (destroyed with the problem)
    std::vector<uint8_t> fixed_host;
    // fine-level PCG vectors
    double *U = nullptr, *F = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr;
    // differentiable forward/backward: filtered FP64 design, dJ/dxPhys, adjoint and saved vectors
    double *xphys64 = nullptr, *dphys = nullptr, *dtmp = nullptr, *lam = nullptr, *usave = nullptr, *fsave = nullptr;
    bool fwd_valid = false;
    tpo_design_opts fwd_opts{};
    double *partials = nullptr;
    size_t npartials = 0;
    CGState *st = nullptr;
    CGState *st_host = nullptr;  // pinned
    double *scal = nullptr;      // device scalars: [0] compliance, [1] change bits
    double *scal_host = nullptr; // pinned
    unsigned *dot_counter = nullptr;
    double *Ttmp = nullptr;
    // FP32 vectors of the mixed-precision inner solve
    float *r32 = nullptr, *z32 = nullptr, *p32 = nullptr, *Ap32 = nullptr, *d32 = nullptr;
    CGState *st32 = nullptr;
    // tensor-core (TF32) fine-level FP32 apply
    TcKe tke;
    int *tc_err = nullptr;
    bool use_tc = false;     // fine-level smoother/residual applies on tensor cores
    bool use_tc_cg = false;  // the CG operator apply too
    int tc_mode = 0;         // operands of the tensor-core apply: 0 TF32, 1 3xTF32, 2 BF16
    int nrhs = 1;            // right-hand sides of the running solve (grid z of its kernels)
    tpo_batch *batch = nullptr;
    // SIMP working arrays (reference element order)
    float *x_dev = nullptr, *xPhys = nullptr, *energy = nullptr, *dc = nullptr, *dcn = nullptr, *xold = nullptr,
          *Hs = nullptr;
    double Hs_rmin = -1.0;
    OCState *oc = nullptr;
    OCState *oc_host = nullptr;
    bool have_E = false;
    bool shapes_tuned = false;  // launch shapes of the structured applies measured
    double *ftmp64 = nullptr;  // scratch of the density-filter transpose export
    double *hx = nullptr, *hl = nullptr, *hg = nullptr;  // staging of the host-array forward / backward
    float *sx = nullptr;                                  // staging of the host-array SIMP step
    uint8_t *spres = nullptr, *svoid = nullptr;
    // the reference's KSP "BDDC" preconditioner: per-DOF sum of local inverse diagonals,
    // subdomain count and coarse (subdomain-corner) mask; rebuilt when the moduli change
    double *bddc_S = nullptr;
    uint8_t *bddc_W = nullptr, *bddc_coarse = nullptr;
    BddcPart bddc_part{};
    long long E_version = 0, bddc_version = -1;
    int bddc_iters = 3;
    // volumetric stress field of the last SIMP step (reference element order) and its maximum
    float *stress = nullptr;
    unsigned long long *stress_max = nullptr;
    int stress_valid = 0;
    // captured PCG iteration chunks
    cudaGraphExec_t gexec[kIterModes] = {};
    int gchunk[kIterModes] = {};
    long long gnodes[kIterModes] = {};
};

namespace {

void batch_free(tpo_problem *P) {
    tpo_batch *B = P->batch;
    if (!B) return;
    dfree(B->U); dfree(B->F); dfree(B->r); dfree(B->z); dfree(B->p); dfree(B->Ap);
    dfree(B->r32); dfree(B->z32); dfree(B->st); dfree(B->partials); dfree(B->scal); dfree(B->dot_counter);
    if (B->st_host) cudaFreeHost(B->st_host);
    if (B->scal_host) cudaFreeHost(B->scal_host);
    for (int li = 0; li < kMaxLevels; li++) {
        dfree(B->Lb[li]); dfree(B->Lx[li]); dfree(B->Lxt[li]); dfree(B->Lres[li]);
        dfree(B->Lb32[li]); dfree(B->Lx32[li]); dfree(B->Lxt32[li]); dfree(B->Lres32[li]);
    }
    delete B;
    P->batch = nullptr;
}

void problem_free(tpo_problem *P) {
    if (!P) return;
    if (P->s) cudaStreamSynchronize(P->s);
    batch_free(P);
    for (auto &ge : P->gexec)
        if (ge) cudaGraphExecDestroy(ge);
    for (int li = 0; li < P->nl; li++) {
        Level &L = P->L[li];
        dfree(L.fixed); dfree(L.E); dfree(L.Eact); dfree(L.invD); dfree(L.Eact32); dfree(L.invD32);
        dfree(L.b); dfree(L.x); dfree(L.xt); dfree(L.res); dfree(L.K);
        dfree(L.b32); dfree(L.x32); dfree(L.xt32); dfree(L.res32);
        dfree(L.Kinv); dfree(L.Lw); dfree(L.Yw); dfree(L.womega);
        if (L.gj) cudaGraphExecDestroy(L.gj);
    }
    dfree(P->U); dfree(P->F); dfree(P->r); dfree(P->z); dfree(P->p); dfree(P->Ap); dfree(P->partials);
    dfree(P->st); dfree(P->scal); dfree(P->dot_counter); dfree(P->Ttmp);
    dfree(P->xphys64); dfree(P->dphys); dfree(P->dtmp); dfree(P->lam); dfree(P->usave); dfree(P->fsave);
    dfree(P->x_dev); dfree(P->xPhys); dfree(P->energy); dfree(P->dc); dfree(P->dcn); dfree(P->xold); dfree(P->Hs);
    dfree(P->oc); dfree(P->ftmp64); dfree(P->hx); dfree(P->hl); dfree(P->hg);
    dfree(P->sx); dfree(P->spres); dfree(P->svoid);
    dfree(P->bddc_S); dfree(P->bddc_W); dfree(P->bddc_coarse); dfree(P->stress); dfree(P->stress_max);
    dfree(P->r32); dfree(P->z32); dfree(P->p32); dfree(P->Ap32); dfree(P->d32); dfree(P->st32); dfree(P->tc_err);
    if (P->st_host) cudaFreeHost(P->st_host);
    if (P->scal_host) cudaFreeHost(P->scal_host);
    if (P->oc_host) cudaFreeHost(P->oc_host);
    if (P->own) cudaStreamDestroy(P->own);
    delete P;
}

// lambda_max(D^-1/2 Ke D^-1/2), D = diag(Ke): cyclic Jacobi rotations on the symmetric 24x24
// matrix until the off-diagonal mass is at rounding level.
double jacobi_kappa(const double *Ke) {
    constexpr int n = 24;
    double a[n][n];
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) a[i][j] = Ke[i * n + j] / std::sqrt(Ke[i * n + i] * Ke[j * n + j]);
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++) off += a[i][j] * a[i][j];
        if (off < 1e-30) break;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) {
                if (std::fabs(a[p][q]) < 1e-300) continue;
                const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < n; k++) {  // columns p, q
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - sn * akq;
                    a[k][q] = sn * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {  // rows p, q
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - sn * aqk;
                    a[q][k] = sn * apk + c * aqk;
                }
            }
    }
    double mx = a[0][0];
    for (int i = 1; i < n; i++) mx = std::max(mx, a[i][i]);
    return mx;
}

void build_levels(tpo_problem *P) {
    const tpo_mg_opts &o = P->mg;
    if (o.nu1 < 0 || o.nu2 < 0 || o.coarse_iters < 0) fail(TPO_BAD_ARG, "negative sweep count");
    if (o.chebyshev && !(o.cheb_ratio > 1.0)) fail(TPO_BAD_ARG, "Chebyshev smoothing needs cheb_ratio > 1");
    P->nl = 1;
    P->L[0].g = P->g;
    int cx = P->g.nelx, cy = P->g.nely, cz = P->g.nelz;
    const int maxl = std::min<int>(std::max(1, o.max_levels), kMaxLevels);
    for (int li = 1; li < maxl; li++) {
        const int nx = cx / 2, ny = cy / 2, nz = cz / 2;
        if (nx < 2 || ny < 2 || nz < 2) break;
        P->L[li].g = make_grid(nx, ny, nz);
        P->nl++;
        cx = nx; cy = ny; cz = nz;
    }
    std::vector<uint8_t> fm = P->fixed_host;
    size_t maxT = 0;
    for (int li = 0; li < P->nl; li++) {
        Level &L = P->L[li];
        const Grid &g = L.g;
        if (li > 0) fm = downsample_fixed(fm, P->L[li - 1].g, g);
        L.dense = li > 0 && g.ndof <= o.galerkin_max_ndof;
        L.fixed = dalloc<uint8_t>((size_t)g.ndof);
        CK(cudaMemcpy(L.fixed, fm.data(), (size_t)g.ndof, cudaMemcpyHostToDevice));
        L.E = dalloc<double>((size_t)g.nel);
        L.Eact = dalloc<double>((size_t)g.nel);
        L.Eact32 = dalloc<float>((size_t)g.nel);
        L.invD = dalloc<double>((size_t)g.ndof);
        L.invD32 = dalloc<float>((size_t)g.ndof);
        L.xt = dalloc<double>((size_t)g.ndof);
        L.res = dalloc<double>((size_t)g.ndof);
        if (li > 0) {
            L.b = dalloc<double>((size_t)g.ndof);
            L.x = dalloc<double>((size_t)g.ndof);
        }
        if (L.dense) {
            L.K = dalloc<double>((size_t)g.ndof * g.ndof);
            if (P->L[li - 1].dense) maxT = std::max(maxT, (size_t)(P->L[li - 1].g.ndof * g.ndof));
        }
    }
    if (maxT) P->Ttmp = dalloc<double>(maxT);
    if (o.coarse_direct) {
        Level &C = P->L[P->nl - 1];
        if (!C.dense)
            fail(TPO_BAD_ARG, "coarse_direct needs a dense coarsest level (ndof <= galerkin_max_ndof); raise "
                              "max_levels or galerkin_max_ndof");
        const size_t nn = (size_t)C.g.ndof * C.g.ndof;
        C.Kinv = dalloc<double>(nn);
        C.Lw = dalloc<double>(nn);
        C.Yw = dalloc<double>(nn);
        // The inverse takes n sweeps between two fixed buffers at every hierarchy update:
        // captured once here (on a private stream) and replayed as one graph launch.
        const int n = (int)C.g.ndof;
        cudaStream_t cs;
        CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            double *src = C.Lw, *dst = C.Yw;
            for (int k = 0; k < n; k++) {
                k_gj_sweep<<<nblk((long long)n * n), 256, 0, cs>>>(src, dst, n, k, C.invD);
                std::swap(src, dst);
            }
            const cudaError_t le = cudaGetLastError();
            e = cudaStreamEndCapture(cs, &graph);
            if (e == cudaSuccess) e = le;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&C.gj, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        CK(e);
    }
    // Jacobi damping per level.  The reference damps every level with omega; under
    // safe_omega a rediscretised level uses min(omega, 1.9 / kappa(Ke)), where
    // kappa(Ke) = lambda_max(diag(Ke)^-1 Ke) bounds lambda_max(D^-1 A) for any moduli
    // (A and D are both sums of E_e Ke over the elements), so the smoother converges and
    // the symmetric V-cycle stays positive definite; dense levels get theirs on the device
    // from a Gershgorin bound at every hierarchy update (k_dense_jacobi_bound).
    const double kappa = (o.safe_omega || o.chebyshev) ? jacobi_kappa(P->Ke) : 0.0;
    for (int li = 0; li < P->nl; li++) {
        Level &L = P->L[li];
        L.omega = o.omega;
        if (o.safe_omega && !L.dense) L.omega = std::min(o.omega, 1.9 / kappa);
        if (o.safe_omega && L.dense) L.womega = dalloc<double>(1);
        if (o.chebyshev && !L.dense) {
            // Chebyshev iteration on [kappa / ratio, kappa] (Adams et al. 2003): theta and
            // delta the interval's centre and half width, sigma = theta / delta, rho_0 =
            // 1 / sigma, rho_k = 1 / (2 sigma - rho_{k-1}); sweep 0 is x += D^-1 r / theta,
            // sweep k adds rho_k rho_{k-1} (x_k - x_{k-1}) + 2 rho_k / delta D^-1 r
            const double lmax = kappa, lmin = kappa / o.cheb_ratio;
            const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin), sigma = theta / delta;
            L.cheb = 1;
            L.cheb_w0 = 1.0 / theta;
            double rho = 1.0 / sigma;
            const int nsw = std::max({o.nu1, o.nu2, o.nu1 + o.coarse_iters, 1}) + 1;
            L.cheb_cd.assign((size_t)nsw, 0.0);
            L.cheb_cr.assign((size_t)nsw, 0.0);
            for (int k = 1; k < nsw; k++) {
                const double rn = 1.0 / (2.0 * sigma - rho);
                L.cheb_cd[k] = rn * rho;
                L.cheb_cr[k] = 2.0 * rn / delta;
                rho = rn;
            }
        }
    }
}

// MGPrecond3D.updateFromFine (:558-582) from densities already on the device.
void build_hierarchy(tpo_problem *P, double Emin);
void tune_apply_shapes(tpo_problem *P);

void set_densities_dev(tpo_problem *P, const float *d_x, double penal, double E0, double Emin) {
    Level &L0 = P->L[0];
    k_evals_fine<<<nblk(L0.g.nel), 256, 0, P->s>>>(d_x, L0.g, penal, E0, Emin, 1, L0.E, L0.Eact, L0.Eact32);
    CKL();
    build_hierarchy(P, Emin);
}

// The same from FP64 densities (the differentiable forward pass).
void set_densities_dev_f64(tpo_problem *P, const double *d_x, double penal, double E0, double Emin) {
    Level &L0 = P->L[0];
    k_evals_fine_f64<<<nblk(L0.g.nel), 256, 0, P->s>>>(d_x, L0.g, penal, E0, Emin, 1, L0.E, L0.Eact, L0.Eact32);
    CKL();
    build_hierarchy(P, Emin);
}

// Fine-level diagonal and every coarse level from the fine moduli in L[0].
void build_hierarchy(tpo_problem *P, double Emin) {
    cudaStream_t s = P->s;
    Level &L0 = P->L[0];
    k_diag<<<nblk(L0.g.nnodes), 256, 0, s>>>(P->ke, L0.g, L0.Eact, L0.fixed, L0.invD, L0.invD32);
    CKL();
    for (int li = 1; li < P->nl; li++) {
        Level &L = P->L[li], &Lf = P->L[li - 1];
        if (L.dense) {
            const long long n = L.g.ndof;
            if (Lf.dense) {
                k_galerkin_T<<<nblk(Lf.g.ndof * n), 256, 0, s>>>(Lf.g, L.g, Lf.K, P->Ttmp);
                CKL();
                k_galerkin_PtT<<<nblk(n * n), 256, 0, s>>>(Lf.g, L.g, P->Ttmp, L.K);
                CKL();
            } else {
                k_galerkin_gather<<<nblk(n * n), 256, 0, s>>>(P->ke, Lf.g, L.g, Lf.Eact, L.K);
                CKL();
            }
            k_dense_invdiag<<<nblk(n), 256, 0, s>>>(L.K, (int)n, L.fixed, L.invD, L.invD32);
            CKL();
            if (L.womega) {
                k_dense_jacobi_bound<<<1, 256, 0, s>>>(L.K, (int)n, L.fixed, P->mg.omega, L.womega);
                CKL();
            }
            if (L.Kinv) {  // coarsest level with a direct solve: explicit inverse by n sweeps
                k_coarse_prepare<<<nblk(n * n), 256, 0, s>>>(L.K, (int)n, L.invD, L.Lw);
                CKL();
                cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
                CK(cudaStreamIsCapturing(s, &cap));
                if (cap == cudaStreamCaptureStatusNone) {
                    CK(cudaGraphLaunch(L.gj, s));  // the n sweeps: Lw -> Yw -> Lw ...
                    g_launches.fetch_add(n);
                } else {  // inside a caller's capture: the sweeps as plain launches
                    double *src = L.Lw, *dst = L.Yw;
                    for (int k = 0; k < (int)n; k++) {
                        k_gj_sweep<<<nblk(n * n), 256, 0, s>>>(src, dst, (int)n, k, L.invD);
                        CKL();
                        std::swap(src, dst);
                    }
                }
                const double *src = (n & 1) ? L.Yw : L.Lw;
                k_coarse_mask_inverse<<<nblk(n * n), 256, 0, s>>>(src, (int)n, L.invD, L.Kinv);
                CKL();
            }
        } else {
            k_evals_avg<<<nblk(L.g.nel), 256, 0, s>>>(Lf.E, Lf.g, L.g, Emin, L.E, L.Eact, L.Eact32);
            CKL();
            k_diag<<<nblk(L.g.nnodes), 256, 0, s>>>(P->ke, L.g, L.Eact, L.fixed, L.invD, L.invD32);
            CKL();
        }
    }
    P->have_E = true;
    P->E_version++;
    if (!P->shapes_tuned) tune_apply_shapes(P);
}

// Launch grid of a solve-path kernel: z = the right-hand sides of a batched solve.
inline dim3 G(const tpo_problem *P, unsigned x) { return dim3(x, 1, (unsigned)P->nrhs); }

// ---- precision-specific buffers ------------------------------------------------------
template <typename T>
struct Prec;
template <>
struct Prec<double> {
    static const double *invD(const Level &L) { return L.invD; }
    static const double *Eact(const Level &L) { return L.Eact; }
    static double *b(Level &L) { return L.b; }
    static double *x(Level &L) { return L.x; }
    static double *xt(Level &L) { return L.xt; }
    static double *res(Level &L) { return L.res; }
    static const WalshKe<double> &ke(const tpo_problem *P) { return P->wk; }
};
template <>
struct Prec<float> {
    static const float *invD(const Level &L) { return L.invD32; }
    static const float *Eact(const Level &L) { return L.Eact32; }
    static float *b(Level &L) { return L.b32; }
    static float *x(Level &L) { return L.x32; }
    static float *xt(Level &L) { return L.xt32; }
    static float *res(Level &L) { return L.res32; }
    static const WalshKe<float> &ke(const tpo_problem *P) { return P->wkf; }
};

// Launch-shape autotuner of the structured apply: on the first hierarchy update every
// structured level times the five best x-chunk counts of the cost model (one warm-up and
// three timed launches each, CUDA events on the problem's stream, zero input) in FP32 and
// FP64 and keeps the fastest; reduction-free launches of the level use it from then on.
template <typename T>
void tune_apply_shape(tpo_problem *P, Level &L) {
    std::vector<int> cand = apply_chunk_candidates<T>(L.g, std::max(apply_conc<T, EpiStore<T>>(), 1));
    if (cand.size() > 5) cand.resize(5);
    if (cand.size() < 2) return;
    const size_t n = (size_t)L.g.ndof;
    T *u = dalloc<T>(n), *o = dalloc<T>(n);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    struct Cleanup {
        T *&u, *&o;
        cudaEvent_t &e0, &e1;
        ~Cleanup() {
            dfree(u);
            dfree(o);
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } cleanup{u, o, e0, e1};
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaMemsetAsync(u, 0, n * sizeof(T), P->s));
    const int idx = sizeof(T) == 8 ? 1 : 0;
    float best_ms = -1.0f;
    int best = 0;
    for (int nch : cand) {
        L.g.nch[idx] = nch;
        EpiStore<T> e{o, nullptr, nullptr, nullptr};
        launch_apply<T>(P->s, L.g, Prec<T>::ke(P), u, Prec<T>::Eact(L), e, nullptr);
        CK(cudaEventRecord(e0, P->s));
        for (int r = 0; r < 3; r++) launch_apply<T>(P->s, L.g, Prec<T>::ke(P), u, Prec<T>::Eact(L), e, nullptr);
        CK(cudaEventRecord(e1, P->s));
        CK(cudaEventSynchronize(e1));
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (best_ms < 0.0f || ms < best_ms) {
            best_ms = ms;
            best = nch;
        }
    }
    L.g.nch[idx] = best;
}
void tune_apply_shapes(tpo_problem *P) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(P->s, &cs));
    if (cs != cudaStreamCaptureStatusNone) return;  // timing needs an uncaptured stream
    for (int li = 0; li < P->nl; li++) {
        Level &L = P->L[li];
        if (L.dense) continue;
        tune_apply_shape<float>(P, L);
        tune_apply_shape<double>(P, L);
    }
    P->g.nch[0] = P->L[0].g.nch[0];  // the fine grid's copy used by the single-apply entries
    P->g.nch[1] = P->L[0].g.nch[1];
    P->shapes_tuned = true;
}

// ---- V-cycle (mgVcycle, assembly/index.ts:837-1048) ------------------------------------
template <typename T>
void smooth_from_zero(tpo_problem *P, int li, const T *b, T *x, const CGState *st) {
    Level &L = P->L[li];
    const long long nvec = (L.g.ndof + 15 / (long long)sizeof(T)) / (16 / (long long)sizeof(T));  // 16-byte vectors
    const T w = (T)(L.cheb ? L.cheb_w0 : L.omega);
    k_smooth0<T><<<G(P, nblk(nvec)), 256, 0, P->s>>>(b, Prec<T>::invD(L), L.fixed, w, L.cheb ? nullptr : L.womega,
                                                    x, L.g.ndof, st);
    CKL();
}
// Sweep number k (0-based) of a smoothing sequence from x into xn.  A Chebyshev level also
// needs to know whether the sequence started at x = 0 (pre-smoothing).
template <typename T>
void smooth(tpo_problem *P, int li, const T *b, const T *x, T *xn, const CGState *st, int k = 0,
            bool from_zero = false) {
    Level &L = P->L[li];
    if (L.dense) {
        const int n = (int)L.g.ndof;
        k_dense_smooth<T><<<G(P, (n + 7) / 8), 256, 0, P->s>>>(L.K, n, x, b, Prec<T>::invD(L), L.fixed, (T)L.omega,
                                                          L.womega, xn, st);
        CKL();
    } else if (L.cheb && k > 0) {
        if (k >= (int)L.cheb_cd.size()) fail(TPO_BAD_ARG, "Chebyshev sweep beyond the level's coefficients");
        EpiCheb<T> e{xn, b, Prec<T>::invD(L), L.fixed, (T)L.cheb_cd[k], (T)L.cheb_cr[k],
                     (from_zero && k == 1) ? 1 : 0, nullptr, nullptr};
        if constexpr (std::is_same_v<T, float>) {
            if (li == 0 && P->use_tc) {
                launch_apply_tc(P->s, L.g, P->tke, x, L.Eact32, e, st, P->tc_err, P->tc_mode, P->nrhs);
                return;
            }
        }
        launch_apply<T>(P->s, L.g, Prec<T>::ke(P), x, Prec<T>::Eact(L), e, st, P->nrhs);
    } else {
        const T w = (T)(L.cheb ? L.cheb_w0 : L.omega);
        EpiSmooth<T> e{xn, b, Prec<T>::invD(L), L.fixed, w, nullptr, nullptr};
        if constexpr (std::is_same_v<T, float>) {
            if (li == 0 && P->use_tc) {
                launch_apply_tc(P->s, L.g, P->tke, x, L.Eact32, e, st, P->tc_err, P->tc_mode, P->nrhs);
                return;
            }
        }
        launch_apply<T>(P->s, L.g, Prec<T>::ke(P), x, Prec<T>::Eact(L), e, st, P->nrhs);
    }
}
template <typename T>
void residual(tpo_problem *P, int li, const T *b, const T *x, T *res, const CGState *st) {
    Level &L = P->L[li];
    if (L.dense) {
        const int n = (int)L.g.ndof;
        k_dense_residual<T><<<G(P, (n + 7) / 8), 256, 0, P->s>>>(L.K, n, x, b, L.fixed, res, st);
        CKL();
    } else {
        EpiResidual<T> e{res, b, L.fixed, nullptr, nullptr};
        if constexpr (std::is_same_v<T, float>) {
            if (li == 0 && P->use_tc) {
                launch_apply_tc(P->s, L.g, P->tke, x, L.Eact32, e, st, P->tc_err, P->tc_mode, P->nrhs);
                return;
            }
        }
        launch_apply<T>(P->s, L.g, Prec<T>::ke(P), x, Prec<T>::Eact(L), e, st, P->nrhs);
    }
}

// x must be treated as zero on entry (it is fully overwritten).
// rdot (level 0 only, may be null): fuse the PCG step r.z / beta into the last sweep of
// an FP64 V-cycle; returns whether it did (not without a post-smoothing sweep).
template <typename T>
bool vcycle(tpo_problem *P, int li, const T *b, T *x, const CGState *st, const double *rdot = nullptr) {
    Level &L = P->L[li];
    const bool last = li == P->nl - 1;
    if (last && L.Kinv) {  // direct coarse solve: x = K^-1 b on the free DOFs
        const int n = (int)L.g.ndof;
        k_dense_mv<T><<<G(P, (n + 7) / 8), 256, 0, P->s>>>(L.Kinv, n, b, x, st);
        CKL();
        return false;
    }
    // Every sweep after the first swaps the two buffers; start in whichever one makes the
    // last sweep land in x, so that no copy is needed at the end.
    const int nswap = std::max(P->mg.nu1 - 1, 0) + (last ? P->mg.coarse_iters : P->mg.nu2);
    T *cur = x, *alt = Prec<T>::xt(L);
    if (nswap & 1) std::swap(cur, alt);
    int nsm = 0;       // sweeps done at this level
    int seq = 0;       // sweeps done in the current smoothing sequence (Chebyshev index)
    bool seq0 = true;  // the current sequence started from x = 0
    auto do_smooth = [&]() {
        if (nsm == 0) {
            smooth_from_zero<T>(P, li, b, cur, st);
        } else {
            smooth<T>(P, li, b, cur, alt, st, seq, seq0);
            std::swap(cur, alt);
        }
        nsm++;
        seq++;
    };
    for (int s = 0; s < P->mg.nu1; s++) do_smooth();
    if (nsm == 0) {
        k_zero<T><<<G(P, nblk(L.g.ndof)), 256, 0, P->s>>>(cur, L.g.ndof, st);
        CKL();
        nsm = 1;  // x is now an explicit zero; later sweeps need the operator
    }
    if (last) {
        // the reference also forms the residual here, but never uses it
        for (int s = 0; s < P->mg.coarse_iters; s++) do_smooth();
    } else {
        Level &C = P->L[li + 1];
        residual<T>(P, li, b, cur, Prec<T>::res(L), st);
        k_restrict<T><<<restrict_grid(C.g, P->nrhs), restrict_block(C.g), 0, P->s>>>(L.g, C.g, Prec<T>::res(L), C.fixed, Prec<T>::b(C), st);
        CKL();
        vcycle<T>(P, li + 1, Prec<T>::b(C), Prec<T>::x(C), st);
        k_prolong<T><<<prolong_grid<T>(L.g, P->nrhs), prolong_block<T>(L.g), 0, P->s>>>(L.g, C.g, Prec<T>::x(C), L.fixed, cur, st);
        CKL();
        seq = 0;  // post-smoothing: a new sequence from the prolonged iterate
        seq0 = false;
        // FP64 only: in the FP32 apply the epilogue's FP64 operands spill registers and the
        // fused sweep costs more than the pass it saves (measured)
        const bool fuse = std::is_same_v<T, double> && rdot && li == 0 && !L.dense && !L.cheb && P->mg.nu2 > 0;
        for (int s = 0; s < P->mg.nu2; s++) {
            if (fuse && s == P->mg.nu2 - 1) {
                // nsm > 0 here: the last sweep is an apply from cur into alt
                CGState *stw = const_cast<CGState *>(st);
                EpiSmoothDot<T> e{alt, b, Prec<T>::invD(L), L.fixed, (T)L.omega, rdot, stw, P->partials,
                                  &stw->counters[3]};
                launch_apply<T>(P->s, L.g, Prec<T>::ke(P), cur, Prec<T>::Eact(L), e, st, P->nrhs);
                std::swap(cur, alt);
                nsm++;
            } else {
                do_smooth();
            }
        }
        if (cur != x) {
            k_copy<T><<<G(P, nblk(L.g.ndof)), 256, 0, P->s>>>(cur, x, L.g.ndof, st);
            CKL();
        }
        return fuse;
    }
    if (cur != x) {
        k_copy<T><<<G(P, nblk(L.g.ndof)), 256, 0, P->s>>>(cur, x, L.g.ndof, st);
        CKL();
    }
    return false;
}

// FP32 buffers of the mixed-precision inner solve, allocated on first use.
void ensure_mixed(tpo_problem *P) {
    if (P->r32) return;
    const size_t nd = (size_t)P->g.ndof;
    P->r32 = dalloc<float>(nd);
    P->z32 = dalloc<float>(nd);
    P->p32 = dalloc<float>(nd);
    P->Ap32 = dalloc<float>(nd);
    P->d32 = dalloc<float>(nd);
    P->st32 = dalloc<CGState>(1);
    CK(cudaMemset(P->st32, 0, sizeof(CGState)));
    P->tc_err = dalloc<int>(1);
    CK(cudaMemset(P->tc_err, 0, sizeof(int)));
    P->tke = make_tc_ke(P->Ke);
    configure_all_tc();
    for (int li = 0; li < P->nl; li++) {
        Level &L = P->L[li];
        const size_t n = (size_t)L.g.ndof;
        L.xt32 = dalloc<float>(n);
        L.res32 = dalloc<float>(n);
        if (li > 0) {
            L.b32 = dalloc<float>(n);
            L.x32 = dalloc<float>(n);
        }
    }
}

// Reliable update of the mixed-precision solve, gated on the device (st32->do_update):
// U += x32, x32 = 0; r = F - K U in FP64 (also written as r32); convergence on the true
// residual.  Both kernels return at once when no update is due.
void reliable_update(tpo_problem *P) {
    Level &L0 = P->L[0];
    const long long n = L0.g.ndof;
    k_rel_merge<<<G(P, red_blocks()), 256, 0, P->s>>>(P->U, P->d32, n, P->st32);
    CKL();
    EpiDefect e{P->r, P->r32, P->F, L0.fixed, P->st32, P->partials, &P->st32->counters[6]};
    launch_apply<double>(P->s, L0.g, P->wk, P->U, L0.Eact, e, nullptr);
}

// ---- PCG ---------------------------------------------------------------------------
// ---- the reference's KSP "BDDC" preconditioner (KSPSolver, js/optimizer-worker-3d.js:1045-1391;
// bddcApply / ebeKSP_BDDC, assembly/index.ts:1204-1517) ------------------------------------
// Partition of KSPSolver._buildSubdomains (:1141-1160): ~8-64 blocks, at least 2 per axis.
BddcPart bddc_partition(const Grid &g) {
    BddcPart bp{};
    const double nx = g.nelx, ny = g.nely, nz = g.nelz;
    const double target = std::max(8.0, std::min(64.0, std::ceil(std::cbrt(nx * ny * nz / 100.0))));
    const double f[3] = {std::round(std::cbrt(target * (nx * nx) / (ny * nz))),
                         std::round(std::cbrt(target * (ny * ny) / (nx * nz))),
                         std::round(std::cbrt(target * (nz * nz) / (nx * ny)))};
    const int nel[3] = {g.nelx, g.nely, g.nelz};
    int *b[3] = {bp.bx, bp.by, bp.bz};
    for (int a = 0; a < 3; a++) {
        bp.ns[a] = std::max(2, (int)std::min(f[a], (double)nel[a]));
        if (bp.ns[a] > kBddcMaxBlocks) fail(TPO_BAD_ARG, "BDDC partition beyond the supported block count");
        for (int k = 0; k <= bp.ns[a]; k++) b[a][k] = (int)std::floor((double)k * nel[a] / bp.ns[a]);
    }
    return bp;
}

// Coarse mask (every DOF of every subdomain's corner nodes, clamped to the grid) and, when
// the moduli changed, the local inverse diagonals (_updateBDDC :1187-1231).
void ensure_bddc(tpo_problem *P) {
    const Grid &g = P->L[0].g;
    if (!P->bddc_S) {
        P->bddc_part = bddc_partition(g);
        const BddcPart &bp = P->bddc_part;
        std::vector<uint8_t> coarse((size_t)g.ndof, 0);
        for (int sz = 0; sz < bp.ns[2]; sz++)
            for (int sy = 0; sy < bp.ns[1]; sy++)
                for (int sx = 0; sx < bp.ns[0]; sx++) {
                    const int x0 = bp.bx[sx], x1 = bp.bx[sx + 1], y0 = bp.by[sy], y1 = bp.by[sy + 1];
                    const int z0 = bp.bz[sz], z1 = bp.bz[sz + 1];
                    if (x1 <= x0 || y1 <= y0 || z1 <= z0) continue;  // empty subdomains are dropped
                    for (int cz : {z0, z1})
                        for (int cy : {y0, y1})
                            for (int cx : {x0, x1}) {
                                const long long node = ((long long)std::min(cx, g.nelx) * g.nny + std::min(cy, g.nely)) *
                                                           g.nnz + std::min(cz, g.nelz);
                                for (int d = 0; d < 3; d++) coarse[(size_t)(3 * node + d)] = 1;
                            }
                }
        P->bddc_S = dalloc<double>((size_t)g.ndof);
        P->bddc_W = dalloc<uint8_t>((size_t)g.ndof);
        P->bddc_coarse = dalloc<uint8_t>((size_t)g.ndof);
        CK(cudaMemcpyAsync(P->bddc_coarse, coarse.data(), (size_t)g.ndof, cudaMemcpyHostToDevice, P->s));
        CK(cudaStreamSynchronize(P->s));
        P->bddc_version = -1;
    }
    if (P->bddc_version != P->E_version) {
        k_bddc_setup<<<nblk(g.nnodes), 256, 0, P->s>>>(P->ke, g, P->L[0].E, P->L[0].fixed, P->bddc_part, P->bddc_S,
                                                       P->bddc_W);
        CKL();
        P->bddc_version = P->E_version;
    }
}

// z = BDDC(r): local step z = S r / W, bddc_iters - 1 undamped Jacobi sweeps z += D^-1 (r -
// K z) with the global diagonal, then the coarse step on the corner DOFs; the sweeps
// ping-pong between z and the fine level's scratch so that the last one lands in z.
void bddc_apply(tpo_problem *P, const double *r, double *z, const CGState *st) {
    Level &L0 = P->L[0];
    const long long n = L0.g.ndof;
    const int napply = std::max(P->bddc_iters, 1);
    double *cur = (napply & 1) ? L0.xt : z, *alt = (napply & 1) ? z : L0.xt;
    k_bddc_local<<<G(P, red_blocks()), 256, 0, P->s>>>(P->bddc_S, P->bddc_W, r, cur, n, st);
    CKL();
    for (int k = 1; k < napply; k++) {
        EpiSmooth<double> e{alt, r, L0.invD, L0.fixed, 1.0, nullptr, nullptr};
        launch_apply<double>(P->s, L0.g, P->wk, cur, L0.Eact, e, st, P->nrhs);
        std::swap(cur, alt);
    }
    EpiBddcCoarse<double> e{alt, r, L0.invD, L0.fixed, P->bddc_coarse, nullptr, nullptr};
    launch_apply<double>(P->s, L0.g, P->wk, cur, L0.Eact, e, st, P->nrhs);
}

void enqueue_iteration(tpo_problem *P, int mode) {
    // mode 0: FP64 MG preconditioner, 1: FP64 Jacobi, 2/3/4: mixed precision (FP32
    // MG-PCG recurrence with FP64 dot products and gated FP64 reliable updates); 3: the
    // fine-level smoother/residual applies on tensor cores; 4: the CG operator as well;
    // 7/8: as 3/4 with 3xTF32; 5/6/9: FP64 PCG with the FP32 V-cycle as preconditioner
    // (6: fine-level V-cycle applies on tensor cores, 9: in 3xTF32)
    Level &L0 = P->L[0];
    const long long n = L0.g.ndof;
    const bool f32_precond = mode == 5 || mode == 6 || mode == 9 || mode == kModeF32Bf16;
    const bool fp32_recurrence = mode == 2 || mode == 3 || mode == 4 || mode == 7 || mode == 8;
    if (f32_precond) {
        EpiCG<double> e{P->Ap, L0.fixed, P->st, P->partials, &P->st->counters[5]};
        launch_apply<double>(P->s, L0.g, P->wk, P->p, L0.Eact, e, P->st, P->nrhs);
        k_cgP_update<<<G(P, red_blocks()), 256, 0, P->s>>>(P->U, P->r, P->r32, P->p, P->Ap, n, P->st, P->partials);
        CKL();
        vcycle<float>(P, 0, P->r32, P->z32, P->st);
        k_cgP_rz<<<G(P, red_blocks()), 256, 0, P->s>>>(P->r, P->z32, L0.fixed, n, P->st, P->partials);
        CKL();
        k_cgP_p<<<G(P, red_blocks()), 256, 0, P->s>>>(P->p, P->z32, n, P->st);
        CKL();
        return;
    }
    if (fp32_recurrence) {
        EpiCG<float> e{P->Ap32, L0.fixed, P->st32, P->partials, &P->st32->counters[5]};
        if (P->use_tc_cg) launch_apply_tc(P->s, L0.g, P->tke, P->p32, L0.Eact32, e, P->st32, P->tc_err, P->tc_mode);
        else launch_apply<float>(P->s, L0.g, P->wkf, P->p32, L0.Eact32, e, P->st32);
        k_cgR_update<float><<<G(P, red_blocks()), 256, 0, P->s>>>(P->d32, P->r32, P->p32, P->Ap32, n, P->st32,
                                                             P->partials);
        CKL();
        reliable_update(P);
        vcycle<float>(P, 0, P->r32, P->z32, P->st32);
        k_cgT_rz<float><<<G(P, red_blocks()), 256, 0, P->s>>>(P->r32, P->z32, L0.fixed, n, P->st32, P->partials);
        CKL();
        k_cgT_p<float><<<G(P, red_blocks()), 256, 0, P->s>>>(P->p32, P->z32, n, P->st32);
        CKL();
        return;
    }
    EpiCG<double> e{P->Ap, L0.fixed, P->st, P->partials, &P->st->counters[5]};
    launch_apply<double>(P->s, L0.g, P->wk, P->p, L0.Eact, e, P->st, P->nrhs);
    if (mode == 0) {
        k_cg_update_mg<<<G(P, red_blocks()), 256, 0, P->s>>>(P->U, P->r, P->p, P->Ap, n, P->st, P->partials);
        CKL();
        if (!vcycle<double>(P, 0, P->r, P->z, P->st, P->r)) {
            k_cg_rz<<<G(P, red_blocks()), 256, 0, P->s>>>(P->r, P->z, L0.fixed, n, P->st, P->partials);
            CKL();
        }
    } else if (mode == kModeBddc) {
        k_cg_update_mg<<<G(P, red_blocks()), 256, 0, P->s>>>(P->U, P->r, P->p, P->Ap, n, P->st, P->partials);
        CKL();
        bddc_apply(P, P->r, P->z, P->st);
        k_cg_rz<<<G(P, red_blocks()), 256, 0, P->s>>>(P->r, P->z, L0.fixed, n, P->st, P->partials);
        CKL();
    } else {
        k_cg_update_jacobi<<<G(P, red_blocks()), 256, 0, P->s>>>(P->U, P->r, P->z, P->p, P->Ap, L0.invD, n, P->st,
                                                             P->partials);
        CKL();
    }
    k_cg_p<<<G(P, red_blocks()), 256, 0, P->s>>>(P->p, P->z, n, P->st);
    CKL();
}

cudaGraphExec_t get_iteration_graph(tpo_problem *P, int mode, int chunk) {
    if (P->gexec[mode] && P->gchunk[mode] == chunk) return P->gexec[mode];
    if (P->gexec[mode]) {
        cudaGraphExecDestroy(P->gexec[mode]);
        P->gexec[mode] = nullptr;
    }
    cudaGraph_t graph;
    const long long before = g_launches.load();
    CK(cudaStreamBeginCapture(P->s, cudaStreamCaptureModeThreadLocal));
    try {
        for (int i = 0; i < chunk; i++) enqueue_iteration(P, mode % kModeStride);
    } catch (...) {
        cudaStreamEndCapture(P->s, &graph);
        cudaGetLastError();
        throw;
    }
    CK(cudaStreamEndCapture(P->s, &graph));
    // captured launches run only when the graph is launched
    P->gnodes[mode] = g_launches.load() - before;
    g_launches.fetch_sub(P->gnodes[mode]);
    cudaGraphExec_t ge;
    CK(cudaGraphInstantiate(&ge, graph, 0));
    cudaGraphDestroy(graph);
    P->gexec[mode] = ge;
    P->gchunk[mode] = chunk;
    return ge;
}

// Replays chunks of captured iterations until the device state says done.
void run_iterations(tpo_problem *P, int mode, CGState *st, CGState *st_host, int max_iter) {
    const int chunk = mode == 1 ? 16 : 4;
    cudaGraphExec_t ge = get_iteration_graph(P, mode, chunk);
    const long long max_launch = (std::max(0, max_iter) + chunk - 1) / chunk + 1;
    for (long long c = 0;; c++) {
        CK(cudaMemcpyAsync(st_host, st, sizeof(CGState) * P->nrhs, cudaMemcpyDeviceToHost, P->s));
        CK(cudaStreamSynchronize(P->s));
        bool all_done = true;
        for (int k = 0; k < P->nrhs; k++) all_done = all_done && st_host[k].done;
        if (all_done) break;
        if (c > max_launch) fail(TPO_CUDA_ERROR, "PCG state machine did not terminate");
        CK(cudaGraphLaunch(ge, P->s));
        g_launches.fetch_add(P->gnodes[mode]);
    }
}

// A tensor-core wait that ran out leaves a flag; report it as TPO_TIMEOUT.
void check_tc_err(tpo_problem *P) {
    if (!P->tc_err) return;
    int h = 0;
    CK(cudaMemcpyAsync(&h, P->tc_err, sizeof(int), cudaMemcpyDeviceToHost, P->s));
    CK(cudaStreamSynchronize(P->s));
    if (h) {
        CK(cudaMemsetAsync(P->tc_err, 0, sizeof(int), P->s));
        fail(TPO_TIMEOUT, "a tensor-core completion wait ran out");
    }
}

double compliance_dev(tpo_problem *P) {
    k_dot<<<G(P, red_blocks()), 256, 0, P->s>>>(P->F, P->U, P->g.ndof, &P->scal[0], P->dot_counter, P->partials);
    CKL();
    CK(cudaMemcpyAsync(P->scal_host, P->scal, sizeof(double) * P->nrhs, cudaMemcpyDeviceToHost, P->s));
    CK(cudaStreamSynchronize(P->s));
    return P->scal_host[0];
}

void solve_fp64(tpo_problem *P, const tpo_solve_opts &o, tpo_solve_info *info) {
    if (!P->have_E) fail(TPO_BAD_ARG, "tpo_solve: densities were never set");
    Level &L0 = P->L[0];
    const long long n = L0.g.ndof;
    const bool f32pre = o.precision == TPO_F32_PRECOND;
    if (f32pre) {
        ensure_mixed(P);
        P->use_tc = o.tensor_cores >= 1;
        P->use_tc_cg = false;
        P->tc_mode = o.tensor_cores >= 5 ? 2 : (o.tensor_cores >= 3 ? 1 : 0);
    }
    if (o.precond == TPO_PREC_BDDC) {
        if (P->nrhs > 1) fail(TPO_BAD_ARG, "the BDDC preconditioner solves one right-hand side at a time");
        if (P->bddc_iters != o.bddc_smoother_iters && P->gexec[kModeBddc]) {  // captured with another count
            cudaGraphExecDestroy(P->gexec[kModeBddc]);
            P->gexec[kModeBddc] = nullptr;
        }
        P->bddc_iters = o.bddc_smoother_iters;
        ensure_bddc(P);
    }
    const int mode = (f32pre ? (P->use_tc ? (P->tc_mode == 1 ? 9 : (P->tc_mode == 2 ? kModeF32Bf16 : 6)) : 5)
                             : (o.precond == TPO_PREC_MG ? 0 : (o.precond == TPO_PREC_BDDC ? kModeBddc : 1))) +
                     (P->nrhs > 1 ? kModeStride : 0);
    const double eps = o.ref_epsilon ? 1e-12 : 0.0;
    k_cg_setup<<<G(P, 1), 32, 0, P->s>>>(P->st, o.tol, o.max_iter, eps);
    CKL();
    if (o.warm_start) {
        k_mask_zero<<<G(P, red_blocks()), 256, 0, P->s>>>(P->U, L0.fixed, n);
        CKL();
        EpiStore<double> es{P->Ap, nullptr, nullptr, nullptr};
        launch_apply<double>(P->s, L0.g, P->wk, P->U, L0.Eact, es, nullptr, P->nrhs);
        k_cg_init_r<<<G(P, red_blocks()), 256, 0, P->s>>>(P->F, P->Ap, L0.fixed, P->U, P->r, n, P->st, P->partials);
    } else {
        k_cg_init_r<<<G(P, red_blocks()), 256, 0, P->s>>>(P->F, nullptr, L0.fixed, P->U, P->r, n, P->st, P->partials);
    }
    CKL();
    if (f32pre) {
        k_cgP_init<<<G(P, red_blocks()), 256, 0, P->s>>>(P->r, P->r32, n);
        CKL();
        vcycle<float>(P, 0, P->r32, P->z32, P->st);
        k_cgP_pz<<<G(P, red_blocks()), 256, 0, P->s>>>(P->r, P->z32, L0.fixed, P->p, n, P->st, P->partials);
    } else {
        if (mode % kModeStride == 0) vcycle<double>(P, 0, P->r, P->z, P->st);
        if (mode % kModeStride == kModeBddc) bddc_apply(P, P->r, P->z, P->st);
        k_cg_pz<<<G(P, red_blocks()), 256, 0, P->s>>>(P->r, P->z, L0.invD, L0.fixed, P->p, n, mode % kModeStride == 1, P->st,
                                                 P->partials);
    }
    CKL();
    run_iterations(P, mode, P->st, P->st_host, o.max_iter);
    const CGState h = *P->st_host;
    P->use_tc = false;
    P->tc_mode = 0;
    if (f32pre) check_tc_err(P);
    const double c = compliance_dev(P);
    if (info) {
        info->iterations = h.iters;
        info->outer_iterations = 1;
        info->converged = h.converged;
        info->rel_residual = h.r0 > 0 ? std::sqrt(h.rr / h.r0) : 0.0;
        info->compliance = c;
    }
    if (h.nonfinite) fail(TPO_NONFINITE, "non-finite residual or step in PCG");
}

// Mixed precision: FP32 MG-preconditioned CG (FP32 vectors, FP32 V-cycle, FP32 or TF32
// tensor-core applies, FP64 dot products) with FP64 defect correction as reliable
// updates: whenever the FP32 recursive residual has dropped by inner_tol since the last
// update, U += x32 and the residual is recomputed in FP64 as r = F - K U, its FP32 copy
// replacing the recursive one; the search direction is kept, so the Krylov space
// survives the correction.  Convergence is decided on the true FP64 residual:
// ||r||^2 < tol^2 ||r0||^2.
void solve_mixed(tpo_problem *P, const tpo_solve_opts &o, tpo_solve_info *info) {
    if (!P->have_E) fail(TPO_BAD_ARG, "tpo_solve: densities were never set");
    ensure_mixed(P);
    P->use_tc = o.tensor_cores >= 1;
    P->use_tc_cg = o.tensor_cores == 2 || o.tensor_cores == 4;
    P->tc_mode = o.tensor_cores >= 3 ? 1 : 0;
    Level &L0 = P->L[0];
    const long long n = L0.g.ndof;
    if (o.warm_start) k_mask_zero<<<G(P, red_blocks()), 256, 0, P->s>>>(P->U, L0.fixed, n);
    else k_zero<double><<<G(P, red_blocks()), 256, 0, P->s>>>(P->U, n, nullptr);
    CKL();
    k_rel_setup<<<G(P, 1), 32, 0, P->s>>>(P->st32, o.tol, o.max_iter, o.inner_tol);
    CKL();
    k_zero<float><<<G(P, red_blocks()), 256, 0, P->s>>>(P->d32, n, nullptr);
    CKL();
    {  // initial residual (do_update starts at 1)
        EpiDefect e{P->r, P->r32, P->F, L0.fixed, P->st32, P->partials, &P->st32->counters[6]};
        launch_apply<double>(P->s, L0.g, P->wk, P->U, L0.Eact, e, nullptr);
    }
    vcycle<float>(P, 0, P->r32, P->z32, P->st32);
    k_cgT_pz<float><<<G(P, red_blocks()), 256, 0, P->s>>>(P->r32, P->z32, L0.fixed, P->p32, n, P->st32, P->partials);
    CKL();
    const int mode = !P->use_tc ? 2 : (P->use_tc_cg ? (P->tc_mode == 1 ? 8 : 4) : (P->tc_mode == 1 ? 7 : 3));
    run_iterations(P, mode, P->st32, P->st_host, o.max_iter);
    const CGState h = *P->st_host;
    P->use_tc = P->use_tc_cg = false;
    P->tc_mode = 0;
    check_tc_err(P);
    const double c = compliance_dev(P);
    P->st_host->converged = h.converged;  // read by the ABI wrappers
    if (info) {
        info->iterations = h.iters;
        info->outer_iterations = h.n_updates;
        info->converged = h.converged;
        info->rel_residual = h.r0 > 0 ? std::sqrt(h.rr / h.r0) : 0.0;
        info->compliance = c;
    }
    if (h.nonfinite) fail(TPO_NONFINITE, "non-finite residual in the mixed-precision solve");
}

void solve_any(tpo_problem *P, const tpo_solve_opts &o, tpo_solve_info *info) {
    if (o.precision == TPO_MIXED) solve_mixed(P, o, info);
    else solve_fp64(P, o, info);
}

tpo_problem *create_problem(const tpo_grid *gr, const double *Ke, double nu, const uint8_t *fixed,
                            const tpo_mg_opts *mg) {
    check_device();
    if (!gr || gr->nelx < 1 || gr->nely < 1 || gr->nelz < 1) fail(TPO_BAD_ARG, "grid must be at least 1x1x1");
    if (!fixed) fail(TPO_BAD_ARG, "fixedMask is null");
    const Grid g = make_grid(gr->nelx, gr->nely, gr->nelz);
    if (g.ndof > (1LL << 31) - 1) fail(TPO_BAD_ARG, "grid too large for 32-bit DOF indices");
    tpo_problem *P = new tpo_problem();
    try {
        P->g = g;
        if (mg) P->mg = *mg;
        else tpo_default_mg_opts(&P->mg);
        if (Ke) std::memcpy(P->Ke, Ke, sizeof P->Ke);
        else device_lk(nu, P->Ke);
        P->ke = make_ke(P->Ke);
        P->kef = make_kef(P->Ke);
        if (!make_walsh_ke(P->Ke, P->wk) || !make_walsh_ke(P->Ke, P->wkf))
            fail(TPO_BAD_ARG, "Ke is not a hex8 matrix of lk()'s form; use the element-list entry points "
                              "(tpo_apply_a_ebe3d / tpo_ebe_pcg) for other element matrices");
        P->fixed_host.assign(fixed, fixed + g.ndof);
        // a blocking stream: ordered with the legacy default stream that callers (torch) use
        CK(cudaStreamCreate(&P->own));
        P->s = P->own;
        build_levels(P);
        {
            Grid gl[kMaxLevels];
            for (int i = 0; i < P->nl; i++) gl[i] = P->L[i].g;
            configure_all_applies(gl, P->nl);
        }
        const size_t nd = (size_t)g.ndof;
        P->U = dalloc<double>(nd);
        P->F = dalloc<double>(nd);
        P->r = dalloc<double>(nd);
        P->z = dalloc<double>(nd);
        P->p = dalloc<double>(nd);
        P->Ap = dalloc<double>(nd);
        CK(cudaMemset(P->U, 0, nd * sizeof(double)));
        CK(cudaMemset(P->F, 0, nd * sizeof(double)));
        // bound on any apply grid (column tiles x up to 512 x-chunks) and on the reductions
        const long long ncol = g.nny * (long long)g.nnz;
        const long long tout = std::min(walsh_out_cols<double>(g.nnz), walsh_out_cols<float>(g.nnz));
        const long long tc_tiles = (long long)((g.nny + kTcNodesY - 1) / kTcNodesY) * ((g.nnz + kTcNodesZ - 1) / kTcNodesZ);
        const size_t colb = (size_t)std::max((ncol + tout - 1) / tout, tc_tiles);
        P->npartials = 2 * std::max<size_t>(4096, colb * (size_t)std::min(g.nnx, 512));
        P->partials = dalloc<double>(P->npartials);
        P->st = dalloc<CGState>(1);
        CK(cudaMemset(P->st, 0, sizeof(CGState)));
        CK(cudaMallocHost(&P->st_host, sizeof(CGState)));
        P->scal = dalloc<double>(4);
        CK(cudaMallocHost(&P->scal_host, 4 * sizeof(double)));
        P->dot_counter = dalloc<unsigned>(1);
        CK(cudaMemset(P->dot_counter, 0, sizeof(unsigned)));
        P->oc = dalloc<OCState>(1);
        CK(cudaMallocHost(&P->oc_host, sizeof(OCState)));
        CK(cudaDeviceSynchronize());
    } catch (...) {
        problem_free(P);
        throw;
    }
    return P;
}

// Sensitivity filter and density filter launches: the shared-memory tiled kernels for
// stencil half-widths up to kFilterMaxHalo, the one-thread-per-element kernels beyond.
void launch_filter_sens(const Grid &g, cudaStream_t s, double rmin, const float *Hs, const float *x, const float *dc,
                        float *dcn) {
    const int R = (int)std::floor(rmin);
    if (R <= kFilterMaxHalo) {
        const int W = 2 * R + 1, T = kFilterTile + 2 * R;
        const size_t smem = (size_t)W * W * W * (sizeof(double) + 2 * sizeof(int)) + 2 * (size_t)T * T * T * sizeof(float);
        const dim3 grid((g.nelx + kFilterTile - 1) / kFilterTile, (g.nely + kFilterTile - 1) / kFilterTile,
                        (g.nelz + kFilterTile - 1) / kFilterTile);
        k_filter_sens_tiled<<<grid, kFilterTile * kFilterTile * kFilterTile, smem, s>>>(g, rmin, Hs, x, dc, dcn);
    } else {
        k_filter_sens<<<nblk(g.nel), 256, 0, s>>>(g, rmin, Hs, x, dc, dcn);
    }
    CKL();
}
// mode 0: the density filter; 1 and 2: the two halves of its transpose (scale, stencil).
void launch_density(const Grid &g, cudaStream_t s, double radius, int mode, const double *in, double *out) {
    const int R = (int)std::ceil(radius);
    if (R <= kFilterMaxHalo) {
        const int W = 2 * R + 1, T = kFilterTile + 2 * R;
        const size_t W3 = (size_t)W * W * W;
        const size_t smem = W3 * sizeof(double) + (W3 + (W3 & 1)) * 2 * sizeof(int) + (size_t)T * T * T * sizeof(double);
        const dim3 grid((g.nelx + kFilterTile - 1) / kFilterTile, (g.nely + kFilterTile - 1) / kFilterTile,
                        (g.nelz + kFilterTile - 1) / kFilterTile);
        k_density_tiled<<<grid, kFilterTile * kFilterTile * kFilterTile, smem, s>>>(g, radius, mode, in, out);
    } else if (mode == 0) {
        k_density_filter<<<nblk(g.nel), 256, 0, s>>>(g, radius, in, out);
    } else if (mode == 1) {
        k_density_scale<<<nblk(g.nel), 256, 0, s>>>(g, radius, in, out);
    } else {
        k_density_stencil<<<nblk(g.nel), 256, 0, s>>>(g, radius, in, out);
    }
    CKL();
}

void ensure_simp_arrays(tpo_problem *P) {
    if (P->xPhys) return;
    const size_t ne = (size_t)P->g.nel;
    P->x_dev = dalloc<float>(ne);
    P->xPhys = dalloc<float>(ne);
    P->energy = dalloc<float>(ne);
    P->dc = dalloc<float>(ne);
    P->dcn = dalloc<float>(ne);
    P->xold = dalloc<float>(ne);
    P->Hs = dalloc<float>(ne);
    P->stress = dalloc<float>(ne);
    P->stress_max = dalloc<unsigned long long>(1);
    CK(cudaMemset(P->stress_max, 0, sizeof(unsigned long long)));
}

// Device state of one OC bisection: stream, bisection state (device and pinned host copy),
// reduction partials and the change scalar.
struct OcCtx {
    cudaStream_t s;
    OCState *oc, *oc_host;
    double *partials, *scal, *scal_host;
    long long n;
};

void run_oc_ctx(const OcCtx &c, const float *d_x, double volfrac, const float *d_dc, const uint8_t *pres,
                const uint8_t *voidm, float *d_xnew, const float *d_xold, double *lmid, int *nb, double *change,
                double move, int max_bisections) {
    k_oc_init<<<1, 32, 0, c.s>>>(c.oc);
    CKL();
    int launched = 0;
    while (launched < max_bisections) {
        const int chunk = std::min(16, max_bisections - launched);
        for (int i = 0; i < chunk; i++) {
            k_oc_step<<<red_blocks(), 256, 0, c.s>>>(d_x, d_dc, pres, voidm, c.n, volfrac, move, c.oc, c.partials);
            CKL();
        }
        launched += chunk;
        CK(cudaMemcpyAsync(c.oc_host, c.oc, sizeof(OCState), cudaMemcpyDeviceToHost, c.s));
        CK(cudaStreamSynchronize(c.s));
        if (c.oc_host->done) break;
    }
    if (!c.oc_host->done)
        fail(TPO_TIMEOUT, "OC bisection did not terminate within " + std::to_string(max_bisections) + " steps");
    unsigned long long *bits = reinterpret_cast<unsigned long long *>(&c.scal[1]);
    CK(cudaMemsetAsync(bits, 0, sizeof(unsigned long long), c.s));
    k_oc_write<<<red_blocks(), 256, 0, c.s>>>(d_x, d_dc, pres, voidm, c.n, move, c.oc, d_xold, d_xnew,
                                              d_xold ? bits : nullptr);
    CKL();
    CK(cudaMemcpyAsync(c.scal_host, c.scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    if (lmid) *lmid = c.oc_host->last_lmid;
    if (nb) *nb = c.oc_host->nb;
    if (change) *change = c.scal_host[1];
}

// OC (js/optimizer-worker-3d.js:3066-3101): device bisection, the host polling every 16
// steps; more than max_bisections steps (the reference's loop ends within ~1100 halvings
// even in degenerate cases) returns TPO_TIMEOUT.
void run_oc(tpo_problem *P, const float *d_x, double volfrac, const float *d_dc, const uint8_t *pres,
            const uint8_t *voidm, float *d_xnew, const float *d_xold, double *lmid, int *nb, double *change,
            double move = 0.2, int max_bisections = 1280) {
    const OcCtx c{P->s, P->oc, P->oc_host, P->partials, P->scal, P->scal_host, P->g.nel};
    run_oc_ctx(c, d_x, volfrac, d_dc, pres, voidm, d_xnew, d_xold, lmid, nb, change, move, max_bisections);
}

void validate_solve_opts(const tpo_solve_opts *o) {
    if (!o) fail(TPO_BAD_ARG, "solve options are null");
    if (o->max_iter < 0) fail(TPO_BAD_ARG, "max_iter < 0");
    if (!(o->tol >= 0)) fail(TPO_BAD_ARG, "tol must be >= 0");
    if (o->precision != TPO_FP64 && o->precision != TPO_MIXED && o->precision != TPO_F32_PRECOND)
        fail(TPO_BAD_ARG, "unknown precision");
    if (o->precond != TPO_PREC_JACOBI && o->precond != TPO_PREC_MG && o->precond != TPO_PREC_BDDC)
        fail(TPO_BAD_ARG, "unknown preconditioner");
    if (o->precision != TPO_FP64 && o->precond != TPO_PREC_MG)
        fail(TPO_BAD_ARG, "the mixed-precision solves use the multigrid preconditioner");
    if (o->precond == TPO_PREC_BDDC && (o->bddc_smoother_iters < 1 || o->bddc_smoother_iters > 64))
        fail(TPO_BAD_ARG, "bddc_smoother_iters must be 1..64");
    if (o->tensor_cores < 0 || o->tensor_cores > 5) fail(TPO_BAD_ARG, "tensor_cores must be 0..5");
    if (o->tensor_cores == 5 && o->precision != TPO_F32_PRECOND)
        fail(TPO_BAD_ARG, "BF16 tensor-core applies (tensor_cores 5) run in the FP32 preconditioner only");
    if (o->precision == TPO_MIXED && !(o->inner_tol > 0 && o->inner_tol < 1))
        fail(TPO_BAD_ARG, "mixed precision needs 0 < inner_tol < 1 (the residual drop between reliable updates)");
}

}  // namespace

// =====================================================================================
// C ABI
// =====================================================================================
extern "C" {

const char *tpo_status_string(tpo_status s) {
    switch (s) {
    case TPO_OK: return "ok";
    case TPO_NOT_CONVERGED: return "not converged";
    case TPO_NONFINITE: return "non-finite value";
    case TPO_OOM: return "out of device memory";
    case TPO_BAD_ARG: return "bad argument";
    case TPO_CUDA_ERROR: return "CUDA error";
    case TPO_NO_DEVICE: return "no usable device";
    case TPO_TIMEOUT: return "bounded wait ran out";
    }
    return "unknown status";
}

const char *tpo_last_error(void) { return g_err.c_str(); }

int64_t tpo_launch_count(void) { return g_launches.load(); }

int tpo_device_available(void) {
    try {
        check_device();
        return 1;
    } catch (...) {
        return 0;
    }
}

tpo_status tpo_lk(double nu, double *Ke576) {
    return guard([&] {
        if (!Ke576) fail(TPO_BAD_ARG, "Ke is null");
        check_device();
        device_lk(nu, Ke576);
    });
}

void tpo_default_mg_opts(tpo_mg_opts *o) {
    if (!o) return;
    o->max_levels = 6;
    o->galerkin_max_ndof = 3000;
    o->nu1 = 2;
    o->nu2 = 2;
    o->omega = 0.5;
    o->coarse_iters = 30;
    o->coarse_direct = 0;
    o->safe_omega = 0;
    o->chebyshev = 0;
    o->cheb_ratio = 16.0;
}

void tpo_default_solve_opts(tpo_solve_opts *o) {
    if (!o) return;
    o->precond = TPO_PREC_MG;
    o->precision = TPO_FP64;
    o->max_iter = 400;
    o->tol = 1e-8;
    o->warm_start = 0;
    o->ref_epsilon = 1;
    o->inner_tol = 0.1;
    o->tensor_cores = 0;
    o->bddc_smoother_iters = 3;
}

tpo_status tpo_create(const tpo_grid *g, const double *Ke, double nu, const uint8_t *fixedMask,
                      const tpo_mg_opts *mg, tpo_problem **out) {
    return guard([&] {
        if (!out) fail(TPO_BAD_ARG, "out is null");
        *out = nullptr;
        *out = create_problem(g, Ke, nu, fixedMask, mg);
    });
}

tpo_status tpo_destroy(tpo_problem *p) {
    return guard([&] { problem_free(p); });
}

tpo_status tpo_sizes(const tpo_problem *p, int64_t *nel, int64_t *ndof, int32_t *levels) {
    return guard([&] {
        if (!p) fail(TPO_BAD_ARG, "problem is null");
        if (nel) *nel = p->g.nel;
        if (ndof) *ndof = p->g.ndof;
        if (levels) *levels = p->nl;
    });
}

tpo_status tpo_level_info(const tpo_problem *p, int32_t level, int32_t *dims) {
    return guard([&] {
        if (!p || !dims) fail(TPO_BAD_ARG, "null argument");
        if (level < 0 || level >= p->nl) fail(TPO_BAD_ARG, "level out of range");
        const Level &L = p->L[level];
        dims[0] = L.g.nelx;
        dims[1] = L.g.nely;
        dims[2] = L.g.nelz;
        dims[3] = (int32_t)L.g.ndof;
        dims[4] = L.dense ? 1 : 0;
    });
}

tpo_status tpo_level_dense(tpo_problem *p, int32_t level, double *K) {
    return guard([&] {
        if (!p || !K) fail(TPO_BAD_ARG, "null argument");
        if (level < 0 || level >= p->nl) fail(TPO_BAD_ARG, "level out of range");
        const Level &L = p->L[level];
        if (!L.dense) fail(TPO_BAD_ARG, "level has no dense operator");
        if (!p->have_E) fail(TPO_BAD_ARG, "densities not set");
        const size_t n = (size_t)L.g.ndof;
        CK(cudaMemcpyAsync(K, L.K, n * n * sizeof(double), cudaMemcpyDeviceToHost, p->s));
        CK(cudaStreamSynchronize(p->s));
    });
}

void *tpo_stream(tpo_problem *p) { return p ? (void *)p->s : nullptr; }

tpo_status tpo_set_stream(tpo_problem *p, void *stream) {
    return guard([&] {
        if (!p) fail(TPO_BAD_ARG, "problem is null");
        CK(cudaStreamSynchronize(p->s));
        p->s = stream ? (cudaStream_t)stream : p->own;
    });
}

tpo_status tpo_set_densities_dev(tpo_problem *p, const float *d_x, double penal, double E0, double Emin) {
    return guard([&] {
        if (!p || !d_x) fail(TPO_BAD_ARG, "null argument");
        set_densities_dev(p, d_x, penal, E0, Emin);
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_set_densities(tpo_problem *p, const float *x, double penal, double E0, double Emin) {
    return guard([&] {
        if (!p || !x) fail(TPO_BAD_ARG, "null argument");
        ensure_simp_arrays(p);
        CK(cudaMemcpyAsync(p->xPhys, x, (size_t)p->g.nel * sizeof(float), cudaMemcpyHostToDevice, p->s));
        set_densities_dev(p, p->xPhys, penal, E0, Emin);
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_set_load(tpo_problem *p, const double *F) {
    return guard([&] {
        if (!p || !F) fail(TPO_BAD_ARG, "null argument");
        CK(cudaMemcpyAsync(p->F, F, (size_t)p->g.ndof * sizeof(double), cudaMemcpyHostToDevice, p->s));
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_set_load_dev(tpo_problem *p, const double *d_F) {
    return guard([&] {
        if (!p || !d_F) fail(TPO_BAD_ARG, "null argument");
        CK(cudaMemcpyAsync(p->F, d_F, (size_t)p->g.ndof * sizeof(double), cudaMemcpyDeviceToDevice, p->s));
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_apply_dev(tpo_problem *p, const double *d_u, double *d_Ku) {
    return guard([&] {
        if (!p || !d_u || !d_Ku) fail(TPO_BAD_ARG, "null argument");
        if (!p->have_E) fail(TPO_BAD_ARG, "densities were never set");
        EpiStore<double> e{d_Ku, nullptr, nullptr, nullptr};
        launch_apply<double>(p->s, p->g, p->wk, d_u, p->L[0].Eact, e, nullptr);
    });
}

tpo_status tpo_apply_f32_dev(tpo_problem *p, const float *d_u, float *d_Ku) {
    return guard([&] {
        if (!p || !d_u || !d_Ku) fail(TPO_BAD_ARG, "null argument");
        if (!p->have_E) fail(TPO_BAD_ARG, "densities were never set");
        EpiStore<float> e{d_Ku, nullptr, nullptr, nullptr};
        launch_apply<float>(p->s, p->g, p->wkf, d_u, p->L[0].Eact32, e, nullptr);
    });
}

tpo_status tpo_apply_tf32_dev(tpo_problem *p, const float *d_u, float *d_Ku) {
    return guard([&] {
        if (!p || !d_u || !d_Ku) fail(TPO_BAD_ARG, "null argument");
        if (!p->have_E) fail(TPO_BAD_ARG, "densities were never set");
        ensure_mixed(p);
        EpiStore<float> e{d_Ku, nullptr, nullptr, nullptr};
        launch_apply_tc(p->s, p->g, p->tke, d_u, p->L[0].Eact32, e, nullptr, p->tc_err, 0);
        check_tc_err(p);
    });
}

tpo_status tpo_apply_3xtf32_dev(tpo_problem *p, const float *d_u, float *d_Ku) {
    return guard([&] {
        if (!p || !d_u || !d_Ku) fail(TPO_BAD_ARG, "null argument");
        if (!p->have_E) fail(TPO_BAD_ARG, "densities were never set");
        ensure_mixed(p);
        EpiStore<float> e{d_Ku, nullptr, nullptr, nullptr};
        launch_apply_tc(p->s, p->g, p->tke, d_u, p->L[0].Eact32, e, nullptr, p->tc_err, 1);
        check_tc_err(p);
    });
}

tpo_status tpo_apply_bf16_dev(tpo_problem *p, const float *d_u, float *d_Ku) {
    return guard([&] {
        if (!p || !d_u || !d_Ku) fail(TPO_BAD_ARG, "null argument");
        if (!p->have_E) fail(TPO_BAD_ARG, "densities were never set");
        ensure_mixed(p);
        EpiStore<float> e{d_Ku, nullptr, nullptr, nullptr};
        launch_apply_tc(p->s, p->g, p->tke, d_u, p->L[0].Eact32, e, nullptr, p->tc_err, 2);
        check_tc_err(p);
    });
}

tpo_status tpo_apply(tpo_problem *p, const double *u, double *Ku) {
    return guard([&] {
        if (!p || !u || !Ku) fail(TPO_BAD_ARG, "null argument");
        if (!p->have_E) fail(TPO_BAD_ARG, "densities were never set");
        const size_t nb = (size_t)p->g.ndof * sizeof(double);
        CK(cudaMemcpyAsync(p->r, u, nb, cudaMemcpyHostToDevice, p->s));
        EpiStore<double> e{p->Ap, nullptr, nullptr, nullptr};
        launch_apply<double>(p->s, p->g, p->wk, p->r, p->L[0].Eact, e, nullptr);
        CK(cudaMemcpyAsync(Ku, p->Ap, nb, cudaMemcpyDeviceToHost, p->s));
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_vcycle(tpo_problem *p, const double *b, double *z) {
    return guard([&] {
        if (!p || !b || !z) fail(TPO_BAD_ARG, "null argument");
        if (!p->have_E) fail(TPO_BAD_ARG, "densities were never set");
        const size_t nb = (size_t)p->g.ndof * sizeof(double);
        CK(cudaMemcpyAsync(p->r, b, nb, cudaMemcpyHostToDevice, p->s));
        vcycle<double>(p, 0, p->r, p->z, nullptr);
        CK(cudaMemcpyAsync(z, p->z, nb, cudaMemcpyDeviceToHost, p->s));
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_solve_dev(tpo_problem *p, const tpo_solve_opts *o, double *d_U, tpo_solve_info *info) {
    tpo_status st = guard([&] {
        if (!p || !d_U) fail(TPO_BAD_ARG, "null argument");
        validate_solve_opts(o);
        const size_t nb = (size_t)p->g.ndof * sizeof(double);
        if (d_U != p->U) CK(cudaMemcpyAsync(p->U, d_U, nb, cudaMemcpyDeviceToDevice, p->s));
        solve_any(p, *o, info);
        if (d_U != p->U) CK(cudaMemcpyAsync(d_U, p->U, nb, cudaMemcpyDeviceToDevice, p->s));
        CK(cudaStreamSynchronize(p->s));
    });
    if (st == TPO_OK && p && p->st_host && !p->st_host->converged) return TPO_NOT_CONVERGED;
    return st;
}

tpo_status tpo_solve(tpo_problem *p, const tpo_solve_opts *o, double *U, tpo_solve_info *info) {
    tpo_status st = guard([&] {
        if (!p || !U) fail(TPO_BAD_ARG, "null argument");
        validate_solve_opts(o);
        const size_t nb = (size_t)p->g.ndof * sizeof(double);
        CK(cudaMemcpyAsync(p->U, U, nb, cudaMemcpyHostToDevice, p->s));
        solve_any(p, *o, info);
        CK(cudaMemcpyAsync(U, p->U, nb, cudaMemcpyDeviceToHost, p->s));
        CK(cudaStreamSynchronize(p->s));
    });
    if (st == TPO_OK && p && p->st_host && !p->st_host->converged) return TPO_NOT_CONVERGED;
    return st;
}

tpo_status tpo_volumetric_snapshot(tpo_problem *p, float *stress, double *max_stress) {
    return guard([&] {
        if (!p || !stress) fail(TPO_BAD_ARG, "null argument");
        if (!p->stress_valid) fail(TPO_BAD_ARG, "no SIMP step has run on this problem");
        unsigned long long bits = 0;
        CK(cudaMemcpyAsync(stress, p->stress, (size_t)p->g.nel * sizeof(float), cudaMemcpyDeviceToHost, p->s));
        CK(cudaMemcpyAsync(&bits, p->stress_max, sizeof(bits), cudaMemcpyDeviceToHost, p->s));
        CK(cudaStreamSynchronize(p->s));
        if (max_stress) {
            double m;
            std::memcpy(&m, &bits, sizeof(m));
            *max_stress = m;
        }
    });
}

tpo_status tpo_get_u(tpo_problem *p, double *U) {
    return guard([&] {
        if (!p || !U) fail(TPO_BAD_ARG, "null argument");
        CK(cudaMemcpyAsync(U, p->U, (size_t)p->g.ndof * sizeof(double), cudaMemcpyDeviceToHost, p->s));
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_element_energy_dev(tpo_problem *p, const double *d_U, float *d_energy) {
    return guard([&] {
        if (!p || !d_U || !d_energy) fail(TPO_BAD_ARG, "null argument");
        k_energy<<<nblk(p->g.nel), 256, 0, p->s>>>(p->ke, p->g, d_U, d_energy);
        CKL();
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_heaviside_dev(tpo_problem *p, const float *d_x, double beta, float *d_xPhys) {
    return guard([&] {
        if (!p || !d_x || !d_xPhys) fail(TPO_BAD_ARG, "null argument");
        k_heaviside<<<nblk(p->g.nel), 256, 0, p->s>>>(d_x, p->g.nel, beta, d_xPhys);
        CKL();
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_sensitivity_dev(tpo_problem *p, const float *d_x, const float *d_xPhys, const float *d_energy,
                               double penal, double E0, double beta, int32_t use_projection, float *d_dc) {
    return guard([&] {
        if (!p || !d_x || !d_xPhys || !d_energy || !d_dc) fail(TPO_BAD_ARG, "null argument");
        k_sensitivity<<<nblk(p->g.nel), 256, 0, p->s>>>(d_x, d_xPhys, d_energy, p->g.nel, penal, E0, beta,
                                                         use_projection, 0, d_dc, 0.0, nullptr, nullptr);
        CKL();
        CK(cudaStreamSynchronize(p->s));
    });
}

static void ensure_hs(tpo_problem *p, double rmin) {
    ensure_simp_arrays(p);
    if (p->Hs_rmin == rmin) return;
    k_filter_hs<<<nblk(p->g.nel), 256, 0, p->s>>>(p->g, rmin, p->Hs);
    CKL();
    p->Hs_rmin = rmin;
}

tpo_status tpo_filter_sens_dev(tpo_problem *p, double rmin, const float *d_x, const float *d_dc, float *d_dcn) {
    return guard([&] {
        if (!p || !d_x || !d_dc || !d_dcn) fail(TPO_BAD_ARG, "null argument");
        if (!(rmin > 0) || rmin > 16) fail(TPO_BAD_ARG, "rmin must be in (0, 16]");
        ensure_hs(p, rmin);
        launch_filter_sens(p->g, p->s, rmin, p->Hs, d_x, d_dc, d_dcn);
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_density_filter_dev(tpo_problem *p, double radius, const double *d_x, double *d_out) {
    return guard([&] {
        if (!p || !d_x || !d_out) fail(TPO_BAD_ARG, "null argument");
        if (!(radius > 0) || radius > 16) fail(TPO_BAD_ARG, "radius must be in (0, 16]");
        launch_density(p->g, p->s, radius, 0, d_x, d_out);
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_density_filter_transpose_dev(tpo_problem *p, double radius, const double *d_g, double *d_out) {
    return guard([&] {
        if (!p || !d_g || !d_out) fail(TPO_BAD_ARG, "null argument");
        if (!(radius > 0) || radius > 16) fail(TPO_BAD_ARG, "radius must be in (0, 16]");
        if (d_g == d_out) fail(TPO_BAD_ARG, "out must not alias the input");
        if (!p->ftmp64) p->ftmp64 = dalloc<double>((size_t)p->g.nel);
        launch_density(p->g, p->s, radius, 1, d_g, p->ftmp64);
        launch_density(p->g, p->s, radius, 2, p->ftmp64, d_out);
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_oc_dev(tpo_problem *p, const float *d_x, double volfrac, const float *d_dc,
                      const uint8_t *d_preserved, const uint8_t *d_void, float *d_xnew, double *lmid,
                      int32_t *bisections) {
    return guard([&] {
        if (!p || !d_x || !d_dc || !d_xnew) fail(TPO_BAD_ARG, "null argument");
        int nb = 0;
        run_oc(p, d_x, volfrac, d_dc, d_preserved, d_void, d_xnew, nullptr, lmid, &nb, nullptr);
        if (bisections) *bisections = nb;
    });
}

tpo_status tpo_oc_update_dev(tpo_problem *p, const float *d_x, const float *d_dc, const uint8_t *d_preserved,
                             const uint8_t *d_void, double volfrac, double move, int32_t max_bisections,
                             float *d_xnew, double *change, double *lmid, int32_t *bisections) {
    return guard([&] {
        if (!p || !d_x || !d_dc || !d_xnew) fail(TPO_BAD_ARG, "null argument");
        if (d_xnew == d_x) fail(TPO_BAD_ARG, "xnew must not alias x (change compares the two)");
        if (!(move >= 0.0)) fail(TPO_BAD_ARG, "move must be >= 0");
        if (max_bisections < 1) fail(TPO_BAD_ARG, "max_bisections must be >= 1");
        int nb = 0;
        double lm = 0.0, ch = 0.0;
        run_oc(p, d_x, volfrac, d_dc, d_preserved, d_void, d_xnew, d_x, &lm, &nb, &ch, move, max_bisections);
        if (change) *change = ch;
        if (lmid) *lmid = lm;
        if (bisections) *bisections = nb;
    });
}

tpo_status tpo_simp_step_dev(tpo_problem *p, const tpo_simp_opts *o, float *d_x, const uint8_t *d_preserved,
                             const uint8_t *d_void, tpo_simp_info *info) {
    return guard([&] {
        if (!p || !o || !d_x) fail(TPO_BAD_ARG, "null argument");
        validate_solve_opts(&o->solve);
        if (!(o->rmin > 0) || o->rmin > 16) fail(TPO_BAD_ARG, "rmin must be in (0, 16]");
        ensure_simp_arrays(p);
        const long long ne = p->g.nel;
        cudaStream_t s = p->s;
        CK(cudaMemcpyAsync(p->xold, d_x, (size_t)ne * sizeof(float), cudaMemcpyDeviceToDevice, s));
        const float *xphys = d_x;
        const double beta = o->use_projection ? o->beta : 1.0;
        if (o->use_projection) {
            k_heaviside<<<nblk(ne), 256, 0, s>>>(d_x, ne, beta, p->xPhys);
            CKL();
            xphys = p->xPhys;
        }
        set_densities_dev(p, xphys, o->penal, o->E0, o->Emin);
        tpo_solve_info si{};
        solve_any(p, o->solve, &si);
        k_energy<<<nblk(ne), 256, 0, s>>>(p->ke, p->g, p->U, p->energy);
        CKL();
        CK(cudaMemsetAsync(p->stress_max, 0, sizeof(unsigned long long), s));
        k_sensitivity<<<nblk(ne), 256, 0, s>>>(d_x, xphys, p->energy, ne, o->penal, o->E0, beta,
                                               o->use_projection, o->guard_sensitivities, p->dc, o->Emin, p->stress,
                                               p->stress_max);
        CKL();
        ensure_hs(p, o->rmin);
        launch_filter_sens(p->g, s, o->rmin, p->Hs, d_x, p->dc, p->dcn);
        p->stress_valid = 1;
        double change = 0;
        run_oc(p, p->xold, o->volfrac, p->dcn, d_preserved, d_void, d_x, p->xold, nullptr, nullptr, &change);
        if (info) {
            info->compliance = si.compliance;
            info->change = change;
            info->cg_iterations = si.iterations;
            info->converged = si.converged;
            info->rel_residual = si.rel_residual;
        }
    });
}

}  // extern "C"

// ---- batched solves ----------------------------------------------------------------------
namespace {
void ensure_batch(tpo_problem *P, int nb, bool f32) {
    if (P->batch && P->batch->nb == nb && (P->batch->f32 || !f32)) return;
    batch_free(P);
    for (int m = kModeStride; m < kIterModes; m++) {  // graphs captured on the previous batch buffers
        if (P->gexec[m]) cudaGraphExecDestroy(P->gexec[m]);
        P->gexec[m] = nullptr;
        P->gchunk[m] = 0;
    }
    tpo_batch *B = new tpo_batch();
    P->batch = B;
    B->nb = nb;
    B->f32 = f32;
    const size_t nd = (size_t)P->g.ndof * nb;
    B->U = dalloc<double>(nd);
    B->F = dalloc<double>(nd);
    B->r = dalloc<double>(nd);
    B->z = dalloc<double>(nd);
    B->p = dalloc<double>(nd);
    B->Ap = dalloc<double>(nd);
    if (f32) {
        B->r32 = dalloc<float>(nd);
        B->z32 = dalloc<float>(nd);
    }
    B->st = dalloc<CGState>(nb);
    CK(cudaMemset(B->st, 0, sizeof(CGState) * nb));
    CK(cudaMallocHost(&B->st_host, sizeof(CGState) * nb));
    B->partials = dalloc<double>(P->npartials * nb);
    B->scal = dalloc<double>(nb);
    CK(cudaMallocHost(&B->scal_host, sizeof(double) * nb));
    B->dot_counter = dalloc<unsigned>(nb);
    CK(cudaMemset(B->dot_counter, 0, sizeof(unsigned) * nb));
    for (int li = 0; li < P->nl; li++) {
        const size_t n = (size_t)P->L[li].g.ndof * nb;
        B->Lxt[li] = dalloc<double>(n);
        B->Lres[li] = dalloc<double>(n);
        if (li > 0) {
            B->Lb[li] = dalloc<double>(n);
            B->Lx[li] = dalloc<double>(n);
        }
        if (f32) {
            B->Lxt32[li] = dalloc<float>(n);
            B->Lres32[li] = dalloc<float>(n);
            if (li > 0) {
                B->Lb32[li] = dalloc<float>(n);
                B->Lx32[li] = dalloc<float>(n);
            }
        }
    }
    CK(cudaDeviceSynchronize());
}

// Exchange the problem's single-right-hand-side buffers with the batch's (twice restores).
void batch_swap(tpo_problem *P) {
    tpo_batch *B = P->batch;
    std::swap(P->U, B->U); std::swap(P->F, B->F); std::swap(P->r, B->r); std::swap(P->z, B->z);
    std::swap(P->p, B->p); std::swap(P->Ap, B->Ap);
    std::swap(P->st, B->st); std::swap(P->st_host, B->st_host); std::swap(P->partials, B->partials);
    std::swap(P->scal, B->scal); std::swap(P->scal_host, B->scal_host); std::swap(P->dot_counter, B->dot_counter);
    if (B->f32) {
        std::swap(P->r32, B->r32);
        std::swap(P->z32, B->z32);
    }
    for (int li = 0; li < P->nl; li++) {
        Level &L = P->L[li];
        std::swap(L.xt, B->Lxt[li]);
        std::swap(L.res, B->Lres[li]);
        if (li > 0) {
            std::swap(L.b, B->Lb[li]);
            std::swap(L.x, B->Lx[li]);
        }
        if (B->f32) {
            std::swap(L.xt32, B->Lxt32[li]);
            std::swap(L.res32, B->Lres32[li]);
            if (li > 0) {
                std::swap(L.b32, B->Lb32[li]);
                std::swap(L.x32, B->Lx32[li]);
            }
        }
    }
    P->nrhs = P->nrhs == 1 ? B->nb : 1;
}
}  // namespace

extern "C" {

tpo_status tpo_solve_multi_dev(tpo_problem *p, const tpo_solve_opts *o, int32_t nrhs, const double *d_F, double *d_U,
                               tpo_solve_info *infos) {
    bool all_conv = true;
    tpo_status st = guard([&] {
        if (!p || !d_F || !d_U) fail(TPO_BAD_ARG, "null argument");
        if (nrhs < 1 || nrhs > 64) fail(TPO_BAD_ARG, "nrhs must be in 1..64");
        validate_solve_opts(o);
        if (o->precond != TPO_PREC_MG || o->precision == TPO_MIXED)
            fail(TPO_BAD_ARG, "batched solves use the multigrid preconditioner in FP64 or TPO_F32_PRECOND");
        if (!p->have_E) fail(TPO_BAD_ARG, "tpo_solve_multi_dev: densities were never set");
        const bool f32 = o->precision == TPO_F32_PRECOND;
        if (f32) ensure_mixed(p);
        ensure_batch(p, nrhs, f32);
        const size_t nb = (size_t)p->g.ndof * nrhs * sizeof(double);
        CK(cudaMemcpyAsync(p->batch->F, d_F, nb, cudaMemcpyDeviceToDevice, p->s));
        CK(cudaMemcpyAsync(p->batch->U, d_U, nb, cudaMemcpyDeviceToDevice, p->s));
        batch_swap(p);
        struct Restore {
            tpo_problem *p;
            ~Restore() {
                if (p->nrhs > 1) batch_swap(p);
            }
        } restore{p};
        tpo_solve_info first{};
        solve_fp64(p, *o, &first);
        CK(cudaMemcpyAsync(d_U, p->U, nb, cudaMemcpyDeviceToDevice, p->s));
        CK(cudaStreamSynchronize(p->s));
        for (int k = 0; k < nrhs; k++) {
            const CGState &h = p->st_host[k];
            all_conv = all_conv && h.converged;
            if (infos) {
                infos[k].iterations = h.iters;
                infos[k].outer_iterations = 1;
                infos[k].converged = h.converged;
                infos[k].rel_residual = h.r0 > 0 ? std::sqrt(h.rr / h.r0) : 0.0;
                infos[k].compliance = p->scal_host[k];
            }
        }
    });
    if (st == TPO_OK && !all_conv) return TPO_NOT_CONVERGED;
    return st;
}

}  // extern "C"

// ---- differentiable forward / backward ---------------------------------------------------
namespace {
void ensure_adjoint(tpo_problem *P) {
    if (P->xphys64) return;
    const size_t ne = (size_t)P->g.nel, nd = (size_t)P->g.ndof;
    P->xphys64 = dalloc<double>(ne);
    P->dphys = dalloc<double>(ne);
    P->dtmp = dalloc<double>(ne);
    P->lam = dalloc<double>(nd);
    P->usave = dalloc<double>(nd);
    P->fsave = dalloc<double>(nd);
}
void validate_design(const tpo_design_opts *d) {
    if (!d) fail(TPO_BAD_ARG, "design options are null");
    if (!(d->penal >= 1.0) || !(d->E0 > 0.0) || !(d->Emin >= 0.0) || !(d->Emin < d->E0))
        fail(TPO_BAD_ARG, "design options need penal >= 1 and 0 <= Emin < E0");
    if (d->filter_radius > 16.0) fail(TPO_BAD_ARG, "filter_radius must be <= 16");
}
double dot_dev(tpo_problem *P, const double *a, const double *b) {
    k_dot<<<red_blocks(), 256, 0, P->s>>>(a, b, P->g.ndof, &P->scal[0], P->dot_counter, P->partials);
    CKL();
    CK(cudaMemcpyAsync(P->scal_host, P->scal, sizeof(double), cudaMemcpyDeviceToHost, P->s));
    CK(cudaStreamSynchronize(P->s));
    return P->scal_host[0];
}
}  // namespace

extern "C" {

tpo_status tpo_set_spring(tpo_problem *p, int64_t dof, double k) {
    return guard([&] {
        if (!p) fail(TPO_BAD_ARG, "null argument");
        if (dof < -1 || dof >= p->g.ndof) fail(TPO_BAD_ARG, "spring DOF out of range");
        if (dof >= 0 && !(k >= 0.0 && std::isfinite(k))) fail(TPO_BAD_ARG, "spring stiffness must be finite and >= 0");
        const double kk = dof >= 0 ? k : 0.0;
        p->g.sdof = p->L[0].g.sdof = dof;
        p->g.sk = p->L[0].g.sk = kk;
        // captured iterations hold the grid by value: capture them again
        for (int m = 0; m < kIterModes; m++) {
            if (p->gexec[m]) cudaGraphExecDestroy(p->gexec[m]);
            p->gexec[m] = nullptr;
            p->gchunk[m] = 0;
        }
        if (p->have_E) {  // the fine-level diagonal includes the spring
            Level &L0 = p->L[0];
            k_diag<<<nblk(L0.g.nnodes), 256, 0, p->s>>>(p->ke, L0.g, L0.Eact, L0.fixed, L0.invD, L0.invD32);
            CKL();
        }
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_forward_dev(tpo_problem *p, const tpo_design_opts *d, const tpo_solve_opts *o, const double *d_x,
                           const double *d_l, double *objective, tpo_solve_info *info) {
    tpo_status st = guard([&] {
        if (!p || !d_x) fail(TPO_BAD_ARG, "null argument");
        validate_design(d);
        validate_solve_opts(o);
        ensure_adjoint(p);
        const long long ne = p->g.nel;
        if (d->filter_radius > 0.0) {
            launch_density(p->g, p->s, d->filter_radius, 0, d_x, p->xphys64);
        } else {
            CK(cudaMemcpyAsync(p->xphys64, d_x, (size_t)ne * sizeof(double), cudaMemcpyDeviceToDevice, p->s));
        }
        set_densities_dev_f64(p, p->xphys64, d->penal, d->E0, d->Emin);
        solve_any(p, *o, info);
        const double J = dot_dev(p, d_l ? d_l : p->F, p->U);
        if (objective) *objective = J;
        p->fwd_valid = true;
        p->fwd_opts = *d;
    });
    if (st == TPO_OK && p && p->st_host && !p->st_host->converged) return TPO_NOT_CONVERGED;
    return st;
}

tpo_status tpo_backward_dev(tpo_problem *p, const tpo_solve_opts *o, const double *d_l, double *d_grad,
                            double *d_grad_phys, tpo_solve_info *info) {
    tpo_status st = guard([&] {
        if (!p || !d_grad) fail(TPO_BAD_ARG, "null argument");
        if (!p->fwd_valid) fail(TPO_BAD_ARG, "tpo_backward_dev needs a preceding tpo_forward_dev");
        validate_solve_opts(o);
        const tpo_design_opts &d = p->fwd_opts;
        const long long ne = p->g.nel;
        const size_t nb = (size_t)p->g.ndof * sizeof(double);
        const double *lam = p->U;  // compliance: self-adjoint
        if (d_l) {  // adjoint solve K lambda = l with the forward solution kept aside
            CK(cudaMemcpyAsync(p->usave, p->U, nb, cudaMemcpyDeviceToDevice, p->s));
            CK(cudaMemcpyAsync(p->fsave, p->F, nb, cudaMemcpyDeviceToDevice, p->s));
            CK(cudaMemcpyAsync(p->F, d_l, nb, cudaMemcpyDeviceToDevice, p->s));
            tpo_solve_opts oa = *o;
            oa.warm_start = 0;
            solve_any(p, oa, info);
            CK(cudaMemcpyAsync(p->lam, p->U, nb, cudaMemcpyDeviceToDevice, p->s));
            CK(cudaMemcpyAsync(p->U, p->usave, nb, cudaMemcpyDeviceToDevice, p->s));
            CK(cudaMemcpyAsync(p->F, p->fsave, nb, cudaMemcpyDeviceToDevice, p->s));
            lam = p->lam;
        } else if (info) {
            *info = tpo_solve_info{0, 0, 1, 0.0, 0.0};
        }
        k_adjoint_sens<<<nblk(ne), 256, 0, p->s>>>(p->ke, p->g, p->xphys64, p->U, lam, d.penal, d.E0, d.Emin,
                                                   p->dphys);
        CKL();
        if (d.filter_radius > 0.0) {
            launch_density(p->g, p->s, d.filter_radius, 1, p->dphys, p->dtmp);
            launch_density(p->g, p->s, d.filter_radius, 2, p->dtmp, d_grad);
        } else {
            CK(cudaMemcpyAsync(d_grad, p->dphys, (size_t)ne * sizeof(double), cudaMemcpyDeviceToDevice, p->s));
        }
        if (d_grad_phys)
            CK(cudaMemcpyAsync(d_grad_phys, p->dphys, (size_t)ne * sizeof(double), cudaMemcpyDeviceToDevice, p->s));
        CK(cudaStreamSynchronize(p->s));
    });
    if (st == TPO_OK && d_l && p && p->st_host && !p->st_host->converged) return TPO_NOT_CONVERGED;
    return st;
}

// Host-array forms of forward / backward / ebeMGPCG for bindings that hold no device
// memory (the Node addon): inputs are staged in device buffers the problem owns.
tpo_status tpo_forward(tpo_problem *p, const tpo_design_opts *d, const tpo_solve_opts *o, const double *x,
                       const double *l, double *objective, tpo_solve_info *info) {
    tpo_status st = guard([&] {
        if (!p || !x) fail(TPO_BAD_ARG, "null argument");
        if (!p->hx) p->hx = dalloc<double>((size_t)p->g.nel);
        CK(cudaMemcpyAsync(p->hx, x, (size_t)p->g.nel * sizeof(double), cudaMemcpyHostToDevice, p->s));
        if (l) {
            if (!p->hl) p->hl = dalloc<double>((size_t)p->g.ndof);
            CK(cudaMemcpyAsync(p->hl, l, (size_t)p->g.ndof * sizeof(double), cudaMemcpyHostToDevice, p->s));
        }
    });
    if (st != TPO_OK) return st;
    return tpo_forward_dev(p, d, o, p->hx, l ? p->hl : nullptr, objective, info);
}

tpo_status tpo_backward(tpo_problem *p, const tpo_solve_opts *o, const double *l, double *grad, tpo_solve_info *info) {
    tpo_status st = guard([&] {
        if (!p || !grad) fail(TPO_BAD_ARG, "null argument");
        if (!p->hg) p->hg = dalloc<double>((size_t)p->g.nel);
        if (l) {
            if (!p->hl) p->hl = dalloc<double>((size_t)p->g.ndof);
            CK(cudaMemcpyAsync(p->hl, l, (size_t)p->g.ndof * sizeof(double), cudaMemcpyHostToDevice, p->s));
        }
    });
    if (st != TPO_OK) return st;
    st = tpo_backward_dev(p, o, l ? p->hl : nullptr, p->hg, nullptr, info);
    if (st != TPO_OK && st != TPO_NOT_CONVERGED) return st;
    const tpo_status c = guard([&] {
        CK(cudaMemcpyAsync(grad, p->hg, (size_t)p->g.nel * sizeof(double), cudaMemcpyDeviceToHost, p->s));
        CK(cudaStreamSynchronize(p->s));
    });
    return c != TPO_OK ? c : st;
}

tpo_status tpo_simp_step(tpo_problem *p, const tpo_simp_opts *o, float *x, const uint8_t *preserved,
                         const uint8_t *voidm, tpo_simp_info *info) {
    tpo_status st = guard([&] {
        if (!p || !x) fail(TPO_BAD_ARG, "null argument");
        const size_t ne = (size_t)p->g.nel;
        if (!p->sx) p->sx = dalloc<float>(ne);
        CK(cudaMemcpyAsync(p->sx, x, ne * sizeof(float), cudaMemcpyHostToDevice, p->s));
        if (preserved) {
            if (!p->spres) p->spres = dalloc<uint8_t>(ne);
            CK(cudaMemcpyAsync(p->spres, preserved, ne, cudaMemcpyHostToDevice, p->s));
        }
        if (voidm) {
            if (!p->svoid) p->svoid = dalloc<uint8_t>(ne);
            CK(cudaMemcpyAsync(p->svoid, voidm, ne, cudaMemcpyHostToDevice, p->s));
        }
    });
    if (st != TPO_OK) return st;
    st = tpo_simp_step_dev(p, o, p->sx, preserved ? p->spres : nullptr, voidm ? p->svoid : nullptr, info);
    if (st != TPO_OK) return st;
    return guard([&] {
        CK(cudaMemcpyAsync(x, p->sx, (size_t)p->g.nel * sizeof(float), cudaMemcpyDeviceToHost, p->s));
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_mgpcg(tpo_problem *p, const double *F, double *U, int32_t maxIter, double tol, int32_t *iters) {
    tpo_status st = tpo_set_load(p, F);
    if (st != TPO_OK) return st;
    tpo_solve_opts o;
    tpo_default_solve_opts(&o);
    o.precond = TPO_PREC_MG;
    o.precision = TPO_FP64;
    o.max_iter = maxIter;
    o.tol = tol;
    o.warm_start = 0;
    o.ref_epsilon = 1;
    tpo_solve_info info{};
    st = tpo_solve(p, &o, U, &info);
    if (iters) *iters = info.iterations;
    return st;
}

tpo_status tpo_ksp_bddc(tpo_problem *p, const double *F, double *U, int32_t maxIter, double tol,
                        int32_t smootherIters, int32_t *iters) {
    tpo_status st = tpo_set_load(p, F);
    if (st != TPO_OK) return st;
    tpo_solve_opts o;
    tpo_default_solve_opts(&o);
    o.precond = TPO_PREC_BDDC;
    o.precision = TPO_FP64;
    o.max_iter = maxIter;
    o.tol = tol;
    o.warm_start = 0;
    o.ref_epsilon = 1;
    o.bddc_smoother_iters = smootherIters;
    tpo_solve_info info{};
    st = tpo_solve(p, &o, U, &info);
    if (iters) *iters = info.iterations;
    return st;
}

}  // extern "C"

// ---- WASM export surface --------------------------------------------------------------
namespace {
struct Csr {
    int64_t *rowptr = nullptr, *cols = nullptr;
    ~Csr() {
        dfree(rowptr);
        dfree(cols);
    }
};

// CSR of (element product slot -> DOF), slots in list order a = 0..count-1, i = 0..es-1.
void build_csr(const int32_t *edofs, int es, const int32_t *elist, int count, int ndof, Csr &c) {
    std::vector<int64_t> rp((size_t)ndof + 1, 0);
    for (int a = 0; a < count; a++) {
        const int e = elist ? elist[a] : a;
        for (int i = 0; i < es; i++) {
            const int d = edofs[(size_t)e * es + i];
            if (d < 0 || d >= ndof) fail(TPO_BAD_ARG, "edof index out of range");
            rp[(size_t)d + 1]++;
        }
    }
    for (int d = 0; d < ndof; d++) rp[d + 1] += rp[d];
    std::vector<int64_t> cols((size_t)rp[ndof]);
    std::vector<int64_t> pos(rp.begin(), rp.end() - 1);
    for (int a = 0; a < count; a++) {
        const int e = elist ? elist[a] : a;
        for (int i = 0; i < es; i++) cols[(size_t)pos[edofs[(size_t)e * es + i]]++] = (int64_t)a * es + i;
    }
    c.rowptr = dalloc<int64_t>(rp.size());
    c.cols = dalloc<int64_t>(cols.size());
    CK(cudaMemcpy(c.rowptr, rp.data(), rp.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
    if (!cols.empty()) CK(cudaMemcpy(c.cols, cols.data(), cols.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
}

template <typename T>
struct DBuf {
    T *p = nullptr;
    explicit DBuf(size_t n) { p = dalloc<T>(n); }
    DBuf(const T *h, size_t n) {
        p = dalloc<T>(n);
        if (n) CK(cudaMemcpy(p, h, n * sizeof(T), cudaMemcpyHostToDevice));
    }
    ~DBuf() { dfree(p); }
};
}  // namespace

extern "C" {

tpo_status tpo_apply_a_ebe3d(const double *Ke, const int32_t *edofs, const double *evals, const int32_t *active,
                             int32_t activeCount, int32_t nel, const double *p, double *Ap, int32_t ndof) {
    return guard([&] {
        if (!Ke || !edofs || !evals || !p || !Ap || (activeCount > 0 && !active)) fail(TPO_BAD_ARG, "null argument");
        if (ndof < 0 || nel < 0 || activeCount < 0) fail(TPO_BAD_ARG, "negative size");
        for (int a = 0; a < activeCount; a++)
            if (active[a] < 0 || active[a] >= nel) fail(TPO_BAD_ARG, "active element index out of range");
        check_device();
        if (ndof == 0) return;
        Csr csr;
        build_csr(edofs, 24, active, activeCount, ndof, csr);
        DBuf<double> dKe(Ke, 576), dE(evals, (size_t)std::max(nel, 1)), dp(p, (size_t)ndof), dAp((size_t)ndof);
        DBuf<int32_t> ded(edofs, (size_t)nel * 24), dact(active, (size_t)std::max(activeCount, 1));
        DBuf<double> y((size_t)std::max(activeCount, 1) * 24);
        if (activeCount > 0) {
            k_elem_products<<<nblk((long long)activeCount * 24), 256>>>(dKe.p, 24, ded.p, dE.p, dact.p, activeCount, 0.0,
                                                                    dp.p, y.p, nullptr);
            CKL();
        }
        k_csr_gather<<<nblk(ndof), 256>>>(csr.rowptr, csr.cols, y.p, ndof, dAp.p, nullptr, nullptr);
        CKL();
        CK(cudaMemcpy(Ap, dAp.p, (size_t)ndof * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

tpo_status tpo_element_energies(const float *U, const float *KE, const int32_t *edofs, int32_t nel,
                                int32_t edofSize, int32_t ndof, float *energies) {
    return guard([&] {
        if (!U || !KE || !edofs || !energies) fail(TPO_BAD_ARG, "null argument");
        if (nel < 0 || ndof < 0 || edofSize < 1 || edofSize > 64) fail(TPO_BAD_ARG, "inconsistent sizes");
        for (long long i = 0; i < (long long)nel * edofSize; i++)
            if (edofs[i] >= ndof) fail(TPO_BAD_ARG, "edof index beyond ndof");
        check_device();
        if (nel == 0) return;
        if (ndof == 0) {  // every index is negative (checked above): all terms are skipped
            std::fill(energies, energies + nel, 0.0f);
            return;
        }
        cudaStream_t s = nullptr;
        CK(cudaStreamCreate(&s));
        struct SG {
            cudaStream_t s;
            ~SG() { cudaStreamDestroy(s); }
        } sg{s};
        DBuf<float> dU(U, (size_t)ndof), dK(KE, (size_t)edofSize * edofSize), dE((size_t)nel);
        DBuf<int32_t> ded(edofs, (size_t)nel * edofSize);
        k_energy_wgsl<<<nblk(nel), 256, 0, s>>>(dU.p, dK.p, ded.p, nel, edofSize, dE.p);
        CKL();
        CK(cudaMemcpyAsync(energies, dE.p, (size_t)nel * sizeof(float), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    });
}

tpo_status tpo_dense_matvec(const double *K, const double *p, double *Ap, int32_t n) {
    return guard([&] {
        if (!K || !p || !Ap) fail(TPO_BAD_ARG, "null argument");
        if (n < 0) fail(TPO_BAD_ARG, "negative size");
        check_device();
        if (n == 0) return;
        DBuf<double> dK(K, (size_t)n * n), dp(p, (size_t)n), dAp((size_t)n);
        k_dense_matvec_seq<<<nblk(n, 128), 128>>>(dK.p, n, dp.p, dAp.p);
        CKL();
        CK(cudaMemcpy(Ap, dAp.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

tpo_status tpo_ebe_pcg(const double *dens, const double *Ke, const int32_t *edofs, const double *F, double *U,
                       const int32_t *freedofs, int32_t nel, int32_t es, int32_t ndof, int32_t nfree, double Emin,
                       double E0, double penal, int32_t maxIter, double tol, int32_t *iters) {
    tpo_status status = TPO_OK;
    tpo_status g = guard([&] {
        if (!dens || !Ke || !edofs || !F || !U || (nfree > 0 && !freedofs)) fail(TPO_BAD_ARG, "null argument");
        if (es != 24 && es != 8) fail(TPO_BAD_ARG, "edofSize must be 24 or 8");
        if (nel < 0 || ndof < 0 || nfree < 0 || nfree > ndof) fail(TPO_BAD_ARG, "inconsistent sizes");
        check_device();
        std::vector<uint8_t> fixed((size_t)ndof, 1);
        for (int i = 0; i < nfree; i++) {
            if (freedofs[i] < 0 || freedofs[i] >= ndof) fail(TPO_BAD_ARG, "freedof out of range");
            fixed[freedofs[i]] = 0;
        }
        const int cgMax = std::min(maxIter, nfree);
        cudaStream_t s = nullptr;
        CK(cudaStreamCreate(&s));
        struct SG {
            cudaStream_t s;
            ~SG() { cudaStreamDestroy(s); }
        } sg{s};
        Csr csr;
        build_csr(edofs, es, nullptr, nel, ndof, csr);
        DBuf<double> dKe(Ke, (size_t)es * es), dd(dens, (size_t)std::max(nel, 1)), dE((size_t)std::max(nel, 1));
        DBuf<int32_t> ded(edofs, (size_t)std::max(nel, 1) * es);
        DBuf<double> dF(F, (size_t)std::max(ndof, 1)), dU(U, (size_t)std::max(ndof, 1));
        DBuf<uint8_t> dfix(fixed.data(), (size_t)std::max(ndof, 1));
        DBuf<double> y((size_t)std::max(nel, 1) * es), invD((size_t)std::max(ndof, 1)), r((size_t)std::max(ndof, 1)),
            z((size_t)std::max(ndof, 1)), pp((size_t)std::max(ndof, 1)), Ap((size_t)std::max(ndof, 1));
        DBuf<CGState> st(1);
        DBuf<double> part(2 * 4096);
        CK(cudaMemsetAsync(st.p, 0, sizeof(CGState), s));
        const double thresh = Emin * 1000.0;
        const unsigned rb = red_blocks();
        if (nel > 0) {
            k_ebe_evals<<<nblk(nel), 256, 0, s>>>(dd.p, nel, Emin, E0, penal, dE.p);
            CKL();
            k_diag_general<<<nblk((long long)nel * es), 256, 0, s>>>(dKe.p, es, ded.p, dE.p, nel, thresh, y.p);
            CKL();
        }
        k_csr_gather<<<nblk(ndof), 256, 0, s>>>(csr.rowptr, csr.cols, y.p, ndof, Ap.p, nullptr, nullptr);
        CKL();
        k_invdiag_general<<<nblk(ndof), 256, 0, s>>>(Ap.p, dfix.p, ndof, invD.p);
        CKL();
        auto apply = [&](const double *in, double *out, const uint8_t *mask, const CGState *cst) {
            if (nel > 0) {
                k_elem_products<<<nblk((long long)nel * es), 256, 0, s>>>(dKe.p, es, ded.p, dE.p, nullptr, nel, thresh,
                                                                           in, y.p, cst);
                CKL();
            }
            k_csr_gather<<<nblk(ndof), 256, 0, s>>>(csr.rowptr, csr.cols, y.p, ndof, out, mask, cst);
            CKL();
        };
        k_cg_setup<<<1, 32, 0, s>>>(st.p, tol, cgMax, 1e-12);
        CKL();
        k_mask_zero<<<rb, 256, 0, s>>>(dU.p, dfix.p, ndof);
        CKL();
        apply(dU.p, Ap.p, nullptr, nullptr);
        k_cg_init_r<<<rb, 256, 0, s>>>(dF.p, Ap.p, dfix.p, dU.p, r.p, ndof, st.p, part.p);
        CKL();
        k_cg_pz<<<rb, 256, 0, s>>>(r.p, z.p, invD.p, dfix.p, pp.p, ndof, 1, st.p, part.p);
        CKL();
        CGState h{};
        const long long max_chunks = (std::max(cgMax, 0) + 15) / 16 + 1;
        for (long long c = 0;; c++) {
            CK(cudaMemcpyAsync(&h, st.p, sizeof(CGState), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            if (h.done) break;
            if (c > max_chunks) fail(TPO_CUDA_ERROR, "PCG state machine did not terminate");
            for (int k = 0; k < 16; k++) {
                apply(pp.p, Ap.p, dfix.p, st.p);
                k_cg_alpha<<<rb, 256, 0, s>>>(pp.p, Ap.p, ndof, st.p, part.p);
                CKL();
                k_cg_update_jacobi<<<rb, 256, 0, s>>>(dU.p, r.p, z.p, pp.p, Ap.p, invD.p, ndof, st.p, part.p);
                CKL();
                k_cg_p<<<rb, 256, 0, s>>>(pp.p, z.p, ndof, st.p);
                CKL();
            }
        }
        CK(cudaMemcpyAsync(U, dU.p, (size_t)ndof * sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (iters) *iters = h.iters;
        if (h.nonfinite) status = TPO_NONFINITE;
        else if (!h.converged) status = TPO_NOT_CONVERGED;
    });
    return g != TPO_OK ? g : status;
}

}  // extern "C"

// ---- the 2D worker (js/optimizer-worker.js, TopologyOptimizerWorker.optimize :347-800) -------
struct tpo_problem2d {
    int nelx = 0, nely = 0, nel = 0, ndof = 0, nfree = 0;
    cudaStream_t s = nullptr;
    double Ke[64];
    Csr csr;
    double *dKe = nullptr, *E = nullptr, *y = nullptr, *invD = nullptr, *r = nullptr, *z = nullptr, *p = nullptr,
           *Ap = nullptr, *U = nullptr, *F = nullptr, *partials = nullptr, *scal = nullptr, *scal_host = nullptr;
    int32_t *edofs = nullptr;
    uint8_t *fixed = nullptr;
    float *xPhys = nullptr, *energy = nullptr, *dc = nullptr, *dcn = nullptr, *xold = nullptr, *Hs = nullptr;
    double Hs_rmin = -1.0;
    CGState *st = nullptr, *st_host = nullptr;
    OCState *oc = nullptr, *oc_host = nullptr;
    unsigned *dot_counter = nullptr;
    // the captured chunk of PCG iterations, for the active-element threshold it was made with
    cudaGraphExec_t gexec = nullptr;
    double gthresh = -1.0;
    long long gnodes = 0;
};

namespace {
void problem2d_free(tpo_problem2d *P) {
    if (!P) return;
    if (P->s) cudaStreamSynchronize(P->s);
    dfree(P->dKe); dfree(P->E); dfree(P->y); dfree(P->invD); dfree(P->r); dfree(P->z); dfree(P->p); dfree(P->Ap);
    dfree(P->U); dfree(P->F); dfree(P->partials); dfree(P->scal); dfree(P->edofs); dfree(P->fixed);
    dfree(P->xPhys); dfree(P->energy); dfree(P->dc); dfree(P->dcn); dfree(P->xold); dfree(P->Hs);
    dfree(P->st); dfree(P->oc); dfree(P->dot_counter);
    if (P->gexec) cudaGraphExecDestroy(P->gexec);
    if (P->st_host) cudaFreeHost(P->st_host);
    if (P->oc_host) cudaFreeHost(P->oc_host);
    if (P->scal_host) cudaFreeHost(P->scal_host);
    if (P->s) cudaStreamDestroy(P->s);
    delete P;
}

// lk() of the 2D worker (:1732-1767): the bilinear quad's 8x8 element matrix for E = 1.
void lk2d(double nu, double *Ke) {
    const double k[8] = {1.0 / 2 - nu / 6, 1.0 / 8 + nu / 8, -1.0 / 4 - nu / 12, -1.0 / 8 + 3 * nu / 8,
                         -1.0 / 4 + nu / 12, -1.0 / 8 - nu / 8, nu / 6, 1.0 / 8 - 3 * nu / 8};
    static const int ord[8][8] = {{0, 1, 2, 3, 4, 5, 6, 7}, {1, 0, 7, 6, 5, 4, 3, 2}, {2, 7, 0, 5, 6, 3, 4, 1},
                                  {3, 6, 5, 0, 7, 2, 1, 4}, {4, 5, 6, 7, 0, 1, 2, 3}, {5, 4, 3, 2, 1, 0, 7, 6},
                                  {6, 3, 4, 1, 2, 7, 0, 5}, {7, 2, 1, 4, 3, 6, 5, 0}};
    const double scale = 1.0 / (1.0 - nu * nu);
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) Ke[i * 8 + j] = k[ord[i][j]] * scale;
}
}  // namespace

extern "C" {

tpo_status tpo_lk2d(double nu, double *Ke64) {
    return guard([&] {
        if (!Ke64) fail(TPO_BAD_ARG, "null argument");
        lk2d(nu, Ke64);
    });
}

tpo_status tpo_create2d(int32_t nelx, int32_t nely, const double *Ke, double nu, const uint8_t *fixedMask,
                        tpo_problem2d **out) {
    return guard([&] {
        if (!out || !fixedMask) fail(TPO_BAD_ARG, "null argument");
        *out = nullptr;
        if (nelx < 1 || nely < 1) fail(TPO_BAD_ARG, "grid dimensions must be positive");
        const long long nel = (long long)nelx * nely, ndof = 2LL * (nelx + 1) * (nely + 1);
        if (ndof > (1LL << 30)) fail(TPO_BAD_ARG, "grid too large for the 2D path");
        check_device();
        std::unique_ptr<tpo_problem2d, void (*)(tpo_problem2d *)> P(new tpo_problem2d(), problem2d_free);
        P->nelx = nelx;
        P->nely = nely;
        P->nel = (int)nel;
        P->ndof = (int)ndof;
        if (Ke) std::memcpy(P->Ke, Ke, sizeof(P->Ke));
        else lk2d(nu, P->Ke);
        CK(cudaStreamCreateWithFlags(&P->s, cudaStreamNonBlocking));
        // _precomputeEdofs2D (:247-268): element idx = ely + elx*nely, node = (nely+1)*x + y
        std::vector<int32_t> ed((size_t)nel * 8);
        for (int ely = 0; ely < nely; ely++)
            for (int elx = 0; elx < nelx; elx++) {
                const size_t o = (size_t)(ely + elx * nely) * 8;
                const int n1 = (nely + 1) * elx + ely, n2 = (nely + 1) * (elx + 1) + ely;
                const int v[8] = {2 * n1, 2 * n1 + 1, 2 * n2, 2 * n2 + 1, 2 * n2 + 2, 2 * n2 + 3, 2 * n1 + 2, 2 * n1 + 3};
                for (int q = 0; q < 8; q++) ed[o + q] = v[q];
            }
        for (long long i = 0; i < ndof; i++) P->nfree += fixedMask[i] ? 0 : 1;
        build_csr(ed.data(), 8, nullptr, (int)nel, (int)ndof, P->csr);
        P->edofs = dalloc<int32_t>(ed.size());
        CK(cudaMemcpy(P->edofs, ed.data(), ed.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
        P->fixed = dalloc<uint8_t>((size_t)ndof);
        CK(cudaMemcpy(P->fixed, fixedMask, (size_t)ndof, cudaMemcpyHostToDevice));
        P->dKe = dalloc<double>(64);
        CK(cudaMemcpy(P->dKe, P->Ke, sizeof(P->Ke), cudaMemcpyHostToDevice));
        for (double **v : {&P->invD, &P->r, &P->z, &P->p, &P->Ap, &P->U, &P->F}) *v = dalloc<double>((size_t)ndof);
        CK(cudaMemset(P->F, 0, (size_t)ndof * sizeof(double)));
        CK(cudaMemset(P->U, 0, (size_t)ndof * sizeof(double)));
        P->E = dalloc<double>((size_t)nel);
        P->y = dalloc<double>((size_t)nel * 8);
        for (float **v : {&P->xPhys, &P->energy, &P->dc, &P->dcn, &P->xold, &P->Hs}) *v = dalloc<float>((size_t)nel);
        P->partials = dalloc<double>(8192);
        P->scal = dalloc<double>(2);
        P->st = dalloc<CGState>(1);
        P->oc = dalloc<OCState>(1);
        CK(cudaMallocHost(&P->st_host, sizeof(CGState)));
        CK(cudaMallocHost(&P->oc_host, sizeof(OCState)));
        CK(cudaMallocHost(&P->scal_host, 2 * sizeof(double)));
        P->dot_counter = dalloc<unsigned>(1);
        CK(cudaMemset(P->dot_counter, 0, sizeof(unsigned)));
        CK(cudaMemset(P->st, 0, sizeof(CGState)));
        CK(cudaMemset(P->oc, 0, sizeof(OCState)));
        *out = P.release();
    });
}

tpo_status tpo_destroy2d(tpo_problem2d *p) {
    return guard([&] { problem2d_free(p); });
}

tpo_status tpo_set_load2d(tpo_problem2d *p, const double *F) {
    return guard([&] {
        if (!p || !F) fail(TPO_BAD_ARG, "null argument");
        CK(cudaMemcpyAsync(p->F, F, (size_t)p->ndof * sizeof(double), cudaMemcpyHostToDevice, p->s));
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_get_u2d(tpo_problem2d *p, double *U) {
    return guard([&] {
        if (!p || !U) fail(TPO_BAD_ARG, "null argument");
        CK(cudaMemcpyAsync(U, p->U, (size_t)p->ndof * sizeof(double), cudaMemcpyDeviceToHost, p->s));
        CK(cudaStreamSynchronize(p->s));
    });
}

tpo_status tpo_simp2d_step_dev(tpo_problem2d *p, const tpo_simp2d_opts *o, float *d_x, const uint8_t *d_preserved,
                               const uint8_t *d_void, tpo_simp2d_info *info) {
    return guard([&] {
        if (!p || !o || !d_x) fail(TPO_BAD_ARG, "null argument");
        if (!(o->rmin > 0) || o->rmin > 16) fail(TPO_BAD_ARG, "rmin must be in (0, 16]");
        if (!(o->cg_tol >= 0) || o->cg_max_iter < 0) fail(TPO_BAD_ARG, "invalid CG tolerance or cap");
        cudaStream_t s = p->s;
        const int ne = p->nel, nd = p->ndof;
        const unsigned rb = red_blocks();
        CK(cudaMemcpyAsync(p->xold, d_x, (size_t)ne * sizeof(float), cudaMemcpyDeviceToDevice, s));
        const float *xphys = d_x;
        const double beta = o->use_projection ? o->beta : 1.0;
        if (o->use_projection) {  // _heavisideProject (:1769-1778)
            k_heaviside<<<nblk(ne), 256, 0, s>>>(d_x, ne, beta, p->xPhys);
            CKL();
            xphys = p->xPhys;
        }
        // FE / solveCG (:1780-1873): E by Math.pow, active E > 1000 Emin, Jacobi diagonal,
        // PCG on the free DOFs from U = 0 with the absolute test ||r||^2 < tol^2 and the
        // shifted alpha / beta, at most min(nfree, cg_max_iter) iterations
        const double thresh = o->Emin * 1000.0;
        k_evals_pow_f32<<<nblk(ne), 256, 0, s>>>(xphys, ne, o->Emin, o->E0, o->penal, p->E);
        CKL();
        k_diag_general<<<nblk((long long)ne * 8), 256, 0, s>>>(p->dKe, 8, p->edofs, p->E, ne, thresh, p->y);
        CKL();
        k_csr_gather<<<nblk(nd), 256, 0, s>>>(p->csr.rowptr, p->csr.cols, p->y, nd, p->Ap, nullptr, nullptr);
        CKL();
        k_invdiag_general<<<nblk(nd), 256, 0, s>>>(p->Ap, p->fixed, nd, p->invD);
        CKL();
        const int cgMax = std::min(o->cg_max_iter, p->nfree);
        k_cg_setup<<<1, 32, 0, s>>>(p->st, o->cg_tol, cgMax, 1e-12);
        CKL();
        k_cg_init_r<<<rb, 256, 0, s>>>(p->F, nullptr, p->fixed, p->U, p->r, nd, p->st, p->partials);
        CKL();
        k_cg_abs_tol<<<1, 32, 0, s>>>(p->st, o->cg_tol);
        CKL();
        k_cg_pz<<<rb, 256, 0, s>>>(p->r, p->z, p->invD, p->fixed, p->p, nd, 1, p->st, p->partials);
        CKL();
        // 16 iterations per launch of one captured graph (its kernels return at once once the
        // state says done); the host reads the state between launches
        if (!p->gexec || p->gthresh != thresh) {
            if (p->gexec) cudaGraphExecDestroy(p->gexec);
            p->gexec = nullptr;
            cudaGraph_t graph;
            const long long before = g_launches.load();
            CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            for (int k = 0; k < 16; k++) {
                k_csr_apply<<<nblk(nd), 256, 0, s>>>(p->dKe, 8, p->edofs, p->E, thresh, p->p, p->csr.rowptr,
                                                     p->csr.cols, nd, p->Ap, p->fixed, p->st);
                k_cg_alpha<<<rb, 256, 0, s>>>(p->p, p->Ap, nd, p->st, p->partials);
                k_cg_update_jacobi<<<rb, 256, 0, s>>>(p->U, p->r, p->z, p->p, p->Ap, p->invD, nd, p->st, p->partials);
                k_cg_p<<<rb, 256, 0, s>>>(p->p, p->z, nd, p->st);
                g_launches.fetch_add(4);
            }
            const cudaError_t le = cudaGetLastError();
            const cudaError_t ce = cudaStreamEndCapture(s, &graph);
            CK(le);
            CK(ce);
            p->gnodes = g_launches.load() - before;
            g_launches.fetch_sub(p->gnodes);  // captured launches run only when the graph is launched
            cudaGraphExec_t ge;
            const cudaError_t ie = cudaGraphInstantiate(&ge, graph, 0);
            cudaGraphDestroy(graph);
            CK(ie);
            p->gexec = ge;
            p->gthresh = thresh;
        }
        CGState h{};
        const long long max_chunks = (std::max(cgMax, 0) + 15) / 16 + 1;
        for (long long c = 0;; c++) {
            CK(cudaMemcpyAsync(p->st_host, p->st, sizeof(CGState), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            h = *p->st_host;
            if (h.done) break;
            if (c > max_chunks) fail(TPO_CUDA_ERROR, "PCG state machine did not terminate");
            CK(cudaGraphLaunch(p->gexec, s));
            g_launches.fetch_add(p->gnodes);
        }
        if (h.nonfinite) fail(TPO_NONFINITE, "non-finite residual in the 2D solve");
        // c = F . U
        k_dot<<<rb, 256, 0, s>>>(p->F, p->U, nd, p->scal, p->dot_counter, p->partials);
        CKL();
        CK(cudaMemcpyAsync(p->scal_host, p->scal, sizeof(double), cudaMemcpyDeviceToHost, s));
        // energies, sensitivities (:633-653), 2D sensitivity filter, OC and change
        k_energy_general<<<nblk(ne), 256, 0, s>>>(p->dKe, 8, p->edofs, p->U, ne, p->energy);
        CKL();
        k_sensitivity<<<nblk(ne), 256, 0, s>>>(d_x, xphys, p->energy, ne, o->penal, o->E0, beta, o->use_projection, 0,
                                               p->dc, 0.0, nullptr, nullptr);
        CKL();
        if (p->Hs_rmin != o->rmin) {
            k_filter_hs2d<<<nblk(ne), 256, 0, s>>>(p->nelx, p->nely, o->rmin, p->Hs);
            CKL();
            p->Hs_rmin = o->rmin;
        }
        k_filter_sens2d<<<nblk(ne), 256, 0, s>>>(p->nelx, p->nely, o->rmin, p->Hs, d_x, p->dc, p->dcn);
        CKL();
        CK(cudaStreamSynchronize(s));
        const double compliance = p->scal_host[0];
        double change = 0.0;
        const OcCtx c{s, p->oc, p->oc_host, p->partials, p->scal, p->scal_host, ne};
        run_oc_ctx(c, p->xold, o->volfrac, p->dcn, d_preserved, d_void, d_x, p->xold, nullptr, nullptr, &change, 0.2,
                   1280);
        if (info) {
            info->compliance = compliance;
            info->change = change;
            info->cg_iterations = h.iters;
        }
    });
}

}  // extern "C"

// ---- allocation-free structured apply ---------------------------------------------------
// tpo_apply_static_dev is for callers that must not allocate device memory while they
// run: an embedding whose own memory pool already holds the device's free memory (a
// cudaMalloc there fails, or makes the pool give memory back), and a host loop with a
// latency budget, where cudaMalloc/cudaFree synchronise the whole device.  Its only
// scratch, the element moduli of the call, is a fixed array compiled into the library.
// There is one such array per device and every call shares it, so two calls on one
// device that overlap on the GPU (two streams, two host threads) race; callers
// serialise them.

// Element moduli of the current call in z-fastest internal order, 0 for elements at or
// below 1000 Emin (the layout of a problem's fine-level Eact).  Every entry a call reads
// is written earlier in the same call, so nothing in it has to start at zero.  Host code
// reaches it only through the address cudaGetSymbolAddress returns.
static __device__ __align__(256) double g_static_eact[TPO_STATIC_MAX_ELEMS];

namespace {

// Own instantiation of the apply kernel: its shared-memory attribute is set below
// without touching the instantiation that problem handles use.
struct EpiStoreStatic : EpiStore<double> {};

// k_evals_fine (kernels.cu) restricted to the thresholded FP64 moduli.
__global__ void k_eact_static(const float *__restrict__ x_ref, Grid g, double penal, double E0, double Emin,
                              double *__restrict__ Eact) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.nel) return;
    const int ez = (int)(t % g.nelz);
    const long long r = t / g.nelz;
    const int ey = (int)(r % g.nely);
    const int ex = (int)(r / g.nely);
    const long long ref = ex + (long long)ey * g.nelx + (long long)ez * g.nelx * g.nely;
    const double e = simp_modulus((double)x_ref[ref], penal, E0, Emin, 1);
    Eact[t] = e > Emin * 1000.0 ? e : 0.0;
}

struct StaticApplyDevice {
    bool ready = false;
    double *eact = nullptr;  // address of g_static_eact on this device
    int smem_optin = 0;      // largest dynamic shared memory one CTA may opt in to
    int num_sms = 0;
};
constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mu;
StaticApplyDevice g_static_dev[kStaticMaxDevices];

// One-time set-up of the current device, run with that device current: the device
// address of the scratch array and the apply kernel's shared-memory limit.  Allocates
// nothing.
// The device check (an sm_100 part) is part of that set-up, so later calls pay no
// cudaGetDeviceProperties and write no process-wide state.
const StaticApplyDevice &static_apply_device() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        fail(TPO_NO_DEVICE, "no CUDA device");
    }
    if (dev < 0 || dev >= kStaticMaxDevices) fail(TPO_BAD_ARG, "device ordinal beyond the static apply's table");
    std::lock_guard<std::mutex> lock(g_static_mu);
    StaticApplyDevice &d = g_static_dev[dev];
    if (!d.ready) {
        int major = 0;
        CK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
        if (major < 10) fail(TPO_NO_DEVICE, "libtpo is built for sm_100a; device " + std::to_string(dev) +
                                                " has compute capability " + std::to_string(major) + ".x");
        double *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_static_eact);
        if (e != cudaSuccess || ptr == nullptr) {
            cudaGetLastError();
            fail(TPO_CUDA_ERROR, std::string("cudaGetSymbolAddress of the static apply scratch: ") +
                                     cudaGetErrorString(e));
        }
        CK(cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        CK(cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaFuncSetAttribute(k_apply_w<double, EpiStoreStatic, false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, d.smem_optin));
        CK(cudaFuncSetAttribute(k_apply_w<double, EpiStoreStatic, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, d.smem_optin));
        d.eact = ptr;
        d.ready = true;
    }
    return d;
}

}  // namespace

extern "C" {

tpo_status tpo_apply_static_dev(int32_t nelx, int32_t nely, int32_t nelz, const double *Ke, const float *d_x,
                                double penal, double E0, double Emin, const double *d_u, double *d_Ku,
                                void *stream) {
    return guard([&] {
        if (!Ke || !d_x || !d_u || !d_Ku) fail(TPO_BAD_ARG, "null argument");
        if (nelx < 1 || nely < 1 || nelz < 1) fail(TPO_BAD_ARG, "grid dimensions must be positive");
        const Grid g = make_grid(nelx, nely, nelz);
        if (g.nel > TPO_STATIC_MAX_ELEMS)
            fail(TPO_BAD_ARG, "grid of " + std::to_string(g.nel) + " elements exceeds the static scratch of " +
                                  std::to_string(TPO_STATIC_MAX_ELEMS) + " elements; use a problem handle");
        WalshKe<double> wk;
        if (!make_walsh_ke(Ke, wk)) fail(TPO_BAD_ARG, "Ke is not a hex8 matrix of lk()'s form");
        const StaticApplyDevice &d = static_apply_device();
        if (walsh_out_cols<double>(g.nnz) <= 0) fail(TPO_BAD_ARG, "grid too deep in z for the apply kernel's tiles");
        const size_t smem = walsh_smem_bytes<double>(g);
        if (smem > (size_t)d.smem_optin) fail(TPO_BAD_ARG, "grid too deep in z for the apply kernel's tiles");
        const int per_sm = wk.general ? apply_per_sm<double, EpiStoreStatic, true>(smem)
                                       : apply_per_sm<double, EpiStoreStatic, false>(smem);
        const ApplyShape s = apply_shape<double>(g, per_sm * d.num_sms);
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        k_eact_static<<<nblk(g.nel), 256, 0, st>>>(d_x, g, penal, E0, Emin, d.eact);
        CKL();
        EpiStoreStatic e;
        e.out = d_Ku;
        e.fixed = nullptr;
        e.partials = nullptr;
        e.counter = nullptr;
        if (wk.general)
            k_apply_w<double, EpiStoreStatic, true><<<s.grid, WTile<double>::NT, s.smem, st>>>(wk, g, d_u, d.eact, s.xchunk, e,
                                                                                      nullptr);
        else
            k_apply_w<double, EpiStoreStatic, false><<<s.grid, WTile<double>::NT, s.smem, st>>>(wk, g, d_u, d.eact, s.xchunk,
                                                                                       e, nullptr);
        CKL();
    });
}

}  // extern "C"
