// Learned tail model: a small MLP that predicts the expeRT log-survival line of a query
// (slope, and the log10 survival fraction at the query's top-score bin, from which the
// intercept follows) from its score histogram.  It stands in for the plain fit where
// the histogram holds too few candidates for a stable fit.  No counterpart in the
// reference, whose tail fit is source/core/expeRT.cpp (ModelTailFit) only.
//
// Network: 132 -> 256 -> 256 -> 2, GELU (erf form) after the two hidden layers.
// Weights and activations are bf16, accumulation fp32 in tensor memory, master weights
// and Adam moments fp32.  Every matrix product, forward and backward, runs on the
// tcgen05 tensor cores through one kernel, k_gemm (D = A * B^T with strided operands
// and a fused epilogue).
//
// Kernels:
//   k_features   histogram row -> 132 bf16 features (128-bin window from the first
//                non-empty bin + 4 scalars), optionally after subsampling the
//                candidates to `keep` (exact sampling without replacement, Floyd's method)
//   k_fit_rows   plain FP64 expeRT fit of arbitrary histogram rows
//   k_gemm       tcgen05 GEMM + epilogue (bias, GELU, GELU', fp32 / bf16 stores)
//   k_loss       weighted squared error or Huber loss on normalised targets, its gradient in bf16
//   k_colsum     bias gradients (column sums, fixed order)
//   k_adam       Adam step on the fp32 master weights + bf16 copies
//   k_predict    de-normalised predictions (slope, log10 survival at the top bin)
//   k_apply      fallback policy: learned e-value for sparse queries, plain fit otherwise

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../include/gicops_b200.h"
#include "gx_device.cuh"
#include "gx_device_scope.cuh"
#include "gx_internal.h"
#include "gx_mma.cuh"

typedef __nv_bfloat16 bf16;

namespace gx {
namespace tail {

constexpr int kIn = GX_TAIL_IN, kHid = GX_TAIL_HIDDEN, kOut = GX_TAIL_OUT, kWin = GX_TAIL_WINDOW;
constexpr size_t kW1 = 0, kB1 = kW1 + (size_t)kHid * kIn, kW2 = kB1 + kHid, kB2 = kW2 + (size_t)kHid * kHid,
                 kW3 = kB2 + kHid, kB3 = kW3 + (size_t)kOut * kHid, kNParam = kB3 + kOut;
static_assert(kNParam == GX_TAIL_NPARAM, "parameter layout");
constexpr int kHist = GX_HIST_BINS;

// ------------------------------------------------------------------------------------
// subsampling RNG: SplitMix64 (Steele, Lea, Flood 2014) and a multiply-high range map
// ------------------------------------------------------------------------------------
__host__ __device__ inline uint64_t splitmix64(uint64_t &s)
{
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// uniform integer in [0, j]
__device__ __forceinline__ uint32_t draw_upto(uint64_t &s, uint32_t j)
{
    return (uint32_t)__umul64hi(splitmix64(s), (uint64_t)j + 1ull);
}

// ------------------------------------------------------------------------------------
// k_features: one warp per sample
// ------------------------------------------------------------------------------------
constexpr int kFeatWarps = 4;
constexpr int kHashSlots = 1024;
constexpr uint32_t kEmpty = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t hslot(uint32_t x) { return (x * 2654435761u) >> 22; }

// inserts x, returns false if it was present
__device__ __forceinline__ bool hash_insert(uint32_t *t, uint32_t x)
{
    uint32_t i = hslot(x);
    while (true) {
        const uint32_t v = t[i];
        if (v == x) return false;
        if (v == kEmpty) { t[i] = x; return true; }
        i = (i + 1) & (kHashSlots - 1);
    }
}

struct FeatArgs {
    const uint32_t *hist;   // [nq][kHist]
    const gx_result *res;   // [nq] (maxhyp)
    const float *prec;      // [nq]
    const int32_t *charge;  // [nq] or null
    const gx_tail_sample *smp;
    uint32_t n, nq;
    bf16 *x;                // [n][kIn]
    uint32_t *sub;          // [n][kHist] or null
    int32_t *sub_cpsms;     // [n] or null
    int32_t *hyp_out;       // [n] or null
    int32_t *err;
};

__global__ void __launch_bounds__(kFeatWarps * 32) k_features(FeatArgs a)
{
    __shared__ uint32_t h[kFeatWarps][kHist];
    __shared__ uint32_t cum[kFeatWarps][kHist];
    __shared__ uint32_t tab[kFeatWarps][kHashSlots];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t i = blockIdx.x * kFeatWarps + w;
    if (i >= a.n) return;
    const gx_tail_sample sp = a.smp[i];
    uint32_t *hw = h[w], *cw = cum[w], *tw = tab[w];
    const int hyp = sp.query < a.nq ? a.res[sp.query].maxhyp : -1;
    if (hyp < 0 || hyp >= kHist || sp.keep > GX_TAIL_MAX_KEEP) {
        if (lane == 0 && a.err) atomicExch(a.err, 1);
        for (int k = lane; k < kIn; k += 32) a.x[(uint64_t)i * kIn + k] = __float2bfloat16_rn(0.0f);
        return;
    }
    const uint32_t *src = a.hist + (uint64_t)sp.query * kHist;
    uint32_t tot = 0;
    for (int b = lane; b < kHist; b += 32) { const uint32_t c = src[b]; hw[b] = c; tot += c; }
#pragma unroll
    for (int o = 16; o; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    __syncwarp();
    uint32_t cs = tot;
    if (sp.keep != 0 && sp.keep < tot) {
        // the top-scoring candidate is always kept; the others are drawn from the rest
        const uint32_t top = hw[hyp] > 0 ? 1u : 0u;
        const uint32_t others = tot - top, k = sp.keep - top;
        // inclusive prefix sum of the "others" histogram: lane l owns bins [26l, 26l+26)
        constexpr int kPer = (kHist + 31) / 32;
        const int b0 = lane * kPer, b1 = min(kHist, b0 + kPer);
        uint32_t part = 0;
        for (int b = b0; b < b1; b++) part += hw[b] - ((b == hyp) ? top : 0u);
        uint32_t incl = part;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        uint32_t run = incl - part;
        for (int b = b0; b < b1; b++) { run += hw[b] - ((b == hyp) ? top : 0u); cw[b] = run; }
        for (int t = lane; t < kHashSlots; t += 32) tw[t] = kEmpty;
        __syncwarp();
        if (lane == 0) {
            // Floyd's sampling (Bentley & Floyd 1987): k distinct ranks of [0, others)
            uint64_t st = sp.seed;
            for (uint32_t j = others - k; j < others; j++) {
                const uint32_t t = draw_upto(st, j);
                if (!hash_insert(tw, t)) hash_insert(tw, j);
            }
        }
        __syncwarp();
        for (int b = lane; b < kHist; b += 32) hw[b] = 0;
        __syncwarp();
        for (int t = lane; t < kHashSlots; t += 32) {
            const uint32_t r = tw[t];
            if (r == kEmpty) continue;
            int lo = 0, hi = kHist - 1;  // first bin with cum > r
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (cw[mid] > r) hi = mid; else lo = mid + 1;
            }
            atomicAdd(&hw[lo], 1u);
        }
        __syncwarp();
        if (lane == 0 && top) hw[hyp] += 1;
        __syncwarp();
        cs = sp.keep;
    }
    // the window starts at the first non-empty bin (0 for an empty histogram)
    int b0 = kHist;
    for (int b = lane; b < kHist; b += 32)
        if (hw[b] != 0) { b0 = b; break; }
#pragma unroll
    for (int o = 16; o; o >>= 1) b0 = min(b0, __shfl_xor_sync(0xffffffffu, b0, o));
    if (b0 == kHist) b0 = 0;
    bf16 *xr = a.x + (uint64_t)i * kIn;
    for (int k = lane; k < kWin; k += 32) {
        const int b = b0 + k;
        const uint32_t c = b < kHist ? hw[b] : 0u;
        xr[k] = __float2bfloat16_rn((float)log10(1.0 + (double)c));
    }
    if (lane == 0) {
        xr[kWin + 0] = __float2bfloat16_rn((float)log10((double)(cs > 0 ? cs : 1u)));
        xr[kWin + 1] = __float2bfloat16_rn((float)((double)a.prec[sp.query] / 1000.0));
        xr[kWin + 2] = __float2bfloat16_rn(a.charge ? (float)a.charge[sp.query] : 0.0f);
        xr[kWin + 3] = __float2bfloat16_rn((float)((double)(hyp - b0) / 100.0));
        if (a.sub_cpsms) a.sub_cpsms[i] = (int32_t)cs;
        if (a.hyp_out) a.hyp_out[i] = hyp;
    }
    if (a.sub)
        for (int b = lane; b < kHist; b += 32) a.sub[(uint64_t)i * kHist + b] = hw[b];
}

// ------------------------------------------------------------------------------------
// k_fit_rows: plain FP64 expeRT fit of histogram rows, one warp per row
// ------------------------------------------------------------------------------------
constexpr int kFitWarps = 4;

__global__ void __launch_bounds__(kFitWarps * 32)
    k_fit_rows(const uint32_t *hist, const int32_t *cpsms, const int32_t *hyp, uint32_t n, double *out)
{
    __shared__ uint32_t h[kFitWarps][kHist];
    __shared__ double sx[kFitWarps][kHist + 2];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t i = blockIdx.x * kFitWarps + w;
    if (i >= n) return;
    for (int b = lane; b < kHist; b += 32) h[w][b] = hist[(uint64_t)i * kHist + b];
    __syncwarp();
    if (lane == 0) {
        gx_result r;
        memset(&r, 0, sizeof(r));
        const int hp = min(max(hyp[i], 0), kHist - 1);
        tail_fit(h[w], cpsms[i], hp, sx[w], r);
        out[2 * (uint64_t)i] = r.slope;
        out[2 * (uint64_t)i + 1] = r.icpt;
    }
}

// ------------------------------------------------------------------------------------
// k_gemm: D[M x N] = A[M x K] * B[N x K]^T on tcgen05, one 128 x NT tile per CTA
// ------------------------------------------------------------------------------------
enum Epi : int { kEpiF32 = 0, kEpiBias = 1, kEpiBiasGelu = 2, kEpiDGelu = 3 };

struct GemmArgs {
    const bf16 *A;
    long long sam, sak;   // A(m, k) = A[m*sam + k*sak]
    const bf16 *B;
    long long sbn, sbk;   // B(n, k) = B[n*sbn + k*sbk]
    int M, N, K, NT;      // NT: N tile, multiple of 16 in [16, 256]
    int epi;
    float *D;             // fp32 output (kEpiF32, kEpiBias, kEpiBiasGelu: pre-activation)
    long long ldd;
    bf16 *H;              // bf16 output (kEpiBiasGelu: GELU(z); kEpiDGelu: acc * GELU'(Z))
    long long ldh;
    const float *bias;    // [N]
    const float *Z;       // kEpiDGelu: pre-activation of the forward pass
    long long ldz;
    int32_t *err;
    uint64_t wait_ns;     // limit of each wait for the tensor core (global-timer nanoseconds)
};

constexpr int kGemmThreads = 256;   // two warps per TMEM lane quarter in the epilogue
constexpr int kKStage = 64;
constexpr int kATileBytes = 128 * kKStage * 2;
constexpr int kBufBytes = kATileBytes + 256 * kKStage * 2;   // one stage: the A tile and a B tile of NT <= 256
// Dynamic shared memory of every k_gemm CTA: two operand stages of at most 48 KB (the next
// k-step's operands are copied in while the tensor core reads the current ones), within a
// request that lets at most two CTAs share an SM, whose 512 TMEM columns then always cover
// their two allocations of at most 256 columns.
constexpr int kGemmSmem = 100 * 1024;
static_assert(2 * kBufBytes <= kGemmSmem, "two operand stages");
// After a wait has given up, the kernel still waits this long for the MMA it issued last
// (it reads the operand tiles and writes the TMEM that the kernel frees afterwards).
constexpr uint64_t kDrainNs = 1000000000ull;

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z)
{
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

// 16-byte asynchronous copy global -> shared of src_bytes (0..16) bytes, the rest zero.
__device__ __forceinline__ void cp_async16(uint8_t *dst, const void *src, uint32_t src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(mma::smem_addr(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Stage rows [r0, r0+R) x k [k0, k0+64) of a strided bf16 matrix into the no-swizzle
// K-major core-matrix layout: 16-byte row (r, kc) at ((kc*(R/8) + r/8)*128 + (r%8)*16).
// Out-of-range rows and k are zero.  A row's 16 bytes that are contiguous and aligned in
// global memory travel by an asynchronous copy (complete after cp_async_wait_all), the
// others (strided operands, unaligned rows) by plain loads and stores.
__device__ __forceinline__ void stage_tile(uint8_t *sm, int R, const bf16 *g, long long sr, long long sk, int r0,
                                           int nr, int k0, int nk)
{
    const int units = R * 8;
    const bool kfast = (sk == 1);
    for (int u = threadIdx.x; u < units; u += kGemmThreads) {
        int r, kc;
        if (kfast) { kc = u & 7; r = u >> 3; }
        else { r = u % R; kc = u / R; }
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        const int kb = kc * 8;
        uint8_t *dst = sm + (kc * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16;
        if (r < nr && kb < nk) {
            const bf16 *p = g + (long long)(r0 + r) * sr + (long long)(k0 + kb) * sk;
            if (kfast && ((reinterpret_cast<uintptr_t>(p) & 15u) == 0)) {
                cp_async16(dst, p, 2u * (uint32_t)min(8, nk - kb));
                continue;
            } else {
                uint16_t e[8];
#pragma unroll
                for (int j = 0; j < 8; j++)
                    e[j] = (kb + j < nk) ? __bfloat16_as_ushort(p[(long long)j * sk]) : (uint16_t)0;
                v.x = e[0] | ((uint32_t)e[1] << 16);
                v.y = e[2] | ((uint32_t)e[3] << 16);
                v.z = e[4] | ((uint32_t)e[5] << 16);
                v.w = e[6] | ((uint32_t)e[7] << 16);
            }
        }
        *reinterpret_cast<uint4 *>(dst) = v;
    }
}

// Sixteen consecutive columns of one row when the whole group is inside the matrix and the
// outputs (and Z) allow 16-byte accesses: the same values as the element-wise epilogue, in
// 16-byte stores (four for fp32, two for bf16).
__device__ __forceinline__ void epilogue16(const GemmArgs &a, int row, int col0, const float (&v)[16])
{
    float z[16];
    if (a.epi == kEpiDGelu) {
        const float4 *zp = reinterpret_cast<const float4 *>(a.Z + (long long)row * a.ldz + col0);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const float4 t = zp[q];
            z[4 * q] = t.x; z[4 * q + 1] = t.y; z[4 * q + 2] = t.z; z[4 * q + 3] = t.w;
        }
    } else {
#pragma unroll
        for (int j = 0; j < 16; j++) z[j] = a.epi == kEpiF32 ? v[j] : v[j] + a.bias[col0 + j];
    }
    if (a.epi != kEpiDGelu) {
        float4 *dp = reinterpret_cast<float4 *>(a.D + (long long)row * a.ldd + col0);
#pragma unroll
        for (int q = 0; q < 4; q++) dp[q] = make_float4(z[4 * q], z[4 * q + 1], z[4 * q + 2], z[4 * q + 3]);
    }
    if (a.epi == kEpiBiasGelu || a.epi == kEpiDGelu) {
        uint32_t h[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const float f0 = a.epi == kEpiBiasGelu ? gelu(z[2 * j]) : v[2 * j] * gelu_grad(z[2 * j]);
            const float f1 = a.epi == kEpiBiasGelu ? gelu(z[2 * j + 1]) : v[2 * j + 1] * gelu_grad(z[2 * j + 1]);
            h[j] = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(f0)) |
                   ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(f1)) << 16);
        }
        uint4 *hp = reinterpret_cast<uint4 *>(a.H + (long long)row * a.ldh + col0);
        hp[0] = make_uint4(h[0], h[1], h[2], h[3]);
        hp[1] = make_uint4(h[4], h[5], h[6], h[7]);
    }
}

__device__ __forceinline__ void epilogue(const GemmArgs &a, int row, int col0, const float (&v)[16])
{
#pragma unroll
    for (int j = 0; j < 16; j++) {
        const int n = col0 + j;
        if (n >= a.N) break;
        float acc = v[j];
        switch (a.epi) {
        case kEpiF32:
            a.D[(long long)row * a.ldd + n] = acc;
            break;
        case kEpiBias:
            a.D[(long long)row * a.ldd + n] = acc + a.bias[n];
            break;
        case kEpiBiasGelu: {
            const float z = acc + a.bias[n];
            a.D[(long long)row * a.ldd + n] = z;
            a.H[(long long)row * a.ldh + n] = __float2bfloat16_rn(gelu(z));
            break;
        }
        default: {
            const float z = a.Z[(long long)row * a.ldz + n];
            a.H[(long long)row * a.ldh + n] = __float2bfloat16_rn(acc * gelu_grad(z));
            break;
        }
        }
    }
}

__global__ void __launch_bounds__(kGemmThreads) k_gemm(GemmArgs a)
{
    extern __shared__ __align__(1024) uint8_t dsm[];
    __shared__ uint64_t bar[2];   // completion of the MMAs that read stage 0 / stage 1
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.y * a.NT;
    const uint32_t ncols = a.NT <= 32 ? 32u : a.NT <= 64 ? 64u : a.NT <= 128 ? 128u : 256u;
    if (warp == 0) mma::tmem_alloc(&tmem_base, ncols);
    if (tid == 0) {
        mma::mbar_init(&bar[0], 1);
        mma::mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    mma::fence_before_sync();
    __syncthreads();
    mma::fence_after_sync();
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = mma::idesc_bf16_f32(128, (uint32_t)a.NT);
    const uint32_t a_lbo = 16 * 128, b_lbo = (uint32_t)(a.NT / 8) * 128;
    const int nks = (a.K + kKStage - 1) / kKStage;
    // stage s of k-step ks: A tile at dsm + s * kBufBytes, B tile after it
    auto stage = [&](int st, int k0) {
        uint8_t *sA = dsm + st * kBufBytes;
        stage_tile(sA, 128, a.A, a.sam, a.sak, m0, a.M - m0, k0, a.K - k0);
        stage_tile(sA + kATileBytes, a.NT, a.B, a.sbn, a.sbk, n0, a.N - n0, k0, a.K - k0);
        cp_async_commit();
    };
    uint32_t ph = 0u;     // bit b: the phase of barrier b that its next wait expects
    uint32_t pend = 0u;   // bit b: an MMA commit on barrier b not yet waited for
    bool ok = true;
    stage(0, 0);
    for (int ks = 0; ks < nks; ks++) {
        const int st = ks & 1;
        cp_async_wait_all();   // this thread's copies of stage st (the only ones in flight)
        mma::fence_smem_to_async();
        __syncthreads();
        if (tid == 0) {
            mma::fence_after_sync();
            const uint32_t sa = mma::smem_addr(dsm + st * kBufBytes), sb = sa + (uint32_t)kATileBytes;
            const int k0 = ks * kKStage;
            const int steps = min(kKStage / 16, (a.K - k0 + 15) / 16);
            for (int s2 = 0; s2 < steps; s2++) {
                const uint64_t da = mma::desc_kmajor(sa + (uint32_t)s2 * 2 * a_lbo, a_lbo, 128);
                const uint64_t db = mma::desc_kmajor(sb + (uint32_t)s2 * 2 * b_lbo, b_lbo, 128);
                mma::mma_bf16(tmem, da, db, idesc, (k0 | s2) != 0);
            }
            mma::mma_commit(&bar[st]);
        }
        pend |= 1u << st;
        if (ks + 1 < nks) {
            // the other stage was read by the MMAs of k-step ks - 1: wait for them, then copy
            // k-step ks + 1 into it while the tensor core works on stage st
            const int o = st ^ 1;
            if (pend & (1u << o)) {
                const bool w = mma::mbar_wait(&bar[o], (ph >> o) & 1u, a.wait_ns);
                if (w) {
                    ph ^= 1u << o;
                    pend &= ~(1u << o);
                }
                if (__syncthreads_or(!w)) {   // uniform: every thread leaves the loop together
                    ok = false;
                    break;
                }
            }
            stage(o, (ks + 1) * kKStage);
        }
    }
    if (ok) {   // the last k-step's MMAs
        const int st = (nks - 1) & 1;
        const bool w = mma::mbar_wait(&bar[st], (ph >> st) & 1u, a.wait_ns);
        if (w) {
            ph ^= 1u << st;
            pend &= ~(1u << st);
        }
        if (__syncthreads_or(!w)) ok = false;
    }
    if (!ok) {
        if (tid == 0 && a.err) atomicExch(a.err, 2);
        // the commits not yet observed (each barrier has at most one), bounded
        for (int b = 0; b < 2; b++)
            if (pend & (1u << b)) mma::mbar_wait(&bar[b], (ph >> b) & 1u, kDrainNs);
        cp_async_wait_all();
    } else {
        mma::fence_after_sync();
        // warps w and w + 4 read the same 32 TMEM lanes (rows), alternate 16-column groups
        const int quarter = warp & 3;
        const int row = m0 + quarter * 32 + lane;
        const uint32_t trow = tmem + ((uint32_t)(quarter * 32) << 16);
        // 16-byte stores need the outputs (and Z) 16-byte aligned at every row
        const bool vec = (a.epi == kEpiDGelu || (((uintptr_t)a.D & 15u) == 0 && (a.ldd & 3) == 0)) &&
                         (a.epi < kEpiBiasGelu || (((uintptr_t)a.H & 15u) == 0 && (a.ldh & 7) == 0)) &&
                         (a.epi != kEpiDGelu || (((uintptr_t)a.Z & 15u) == 0 && (a.ldz & 3) == 0));
        for (int c = 16 * (warp >> 2); c < a.NT; c += 32) {
            float v[16];
            mma::tmem_ld16(trow + (uint32_t)c, v);
            if (row < a.M) {
                if (vec && n0 + c + 16 <= a.N) epilogue16(a, row, n0 + c, v);
                else epilogue(a, row, n0 + c, v);
            }
        }
    }
    mma::fence_before_sync();
    __syncthreads();
    if (warp == 0) mma::tmem_dealloc(tmem, ncols);
}

// ------------------------------------------------------------------------------------
// small kernels
// ------------------------------------------------------------------------------------
// loss = sum_i sum_o w_o rho(y_io - t'_io) / n with t' = (t - mean_o) / std_o and dY its
// gradient in bf16.  rho(d) = d^2 (huber = 0), or Huber's loss with that delta:
// d^2 / (2 huber) for |d| < huber, |d| - huber / 2 beyond (gradient d / huber, then +-1).
__global__ void k_loss(const float *Y, const float *T, uint32_t n, const float *norm, float w0, float w1,
                       float huber, bf16 *dY, float *loss)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (i < n) {
        const float w[2] = {w0, w1};
#pragma unroll
        for (int o = 0; o < 2; o++) {
            const float t = (T[2 * (size_t)i + o] - norm[2 * o]) / norm[2 * o + 1];
            const float d = Y[2 * (size_t)i + o] - t;
            float g;
            if (huber > 0.0f) {
                const float ad = fabsf(d);
                if (ad < huber) {
                    l += w[o] * (0.5f * d * d / huber);
                    g = w[o] * d / huber;
                } else {
                    l += w[o] * (ad - 0.5f * huber);
                    g = d > 0.0f ? w[o] : -w[o];
                }
            } else {
                l += w[o] * d * d;
                g = 2.0f * w[o] * d;
            }
            dY[2 * (size_t)i + o] = __float2bfloat16_rn(g / (float)n);
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, l / (float)n);
}

// out[c] = sum over rows r (in order) of X[r*ld + c]
__global__ void k_colsum(const bf16 *X, long long ld, uint32_t rows, uint32_t cols, float *out)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.0f;
    for (uint32_t r = 0; r < rows; r++) s += __bfloat162float(X[(size_t)r * ld + c]);
    out[c] = s;
}

__global__ void k_adam(float *P, const float *G, float *m1, float *m2, bf16 *Pb, uint32_t n, float lr, float b1,
                       float b2, float eps, float bc1, float bc2)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = G[i];
    const float m = b1 * m1[i] + (1.0f - b1) * g;
    const float v = b2 * m2[i] + (1.0f - b2) * g * g;
    m1[i] = m;
    m2[i] = v;
    const float p = P[i] - lr * (m / bc1) / (sqrtf(v / bc2) + eps);
    P[i] = p;
    Pb[i] = __float2bfloat16_rn(p);
}

__global__ void k_to_bf16(const float *P, bf16 *Pb, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) Pb[i] = __float2bfloat16_rn(P[i]);
}

// pred[i] = (slope, log10 survival fraction at the top bin), de-normalised
__global__ void k_predict(const float *Y, uint32_t n, const float *norm, float *pred)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pred[2 * (size_t)i] = Y[2 * (size_t)i] * norm[1] + norm[0];
    pred[2 * (size_t)i + 1] = Y[2 * (size_t)i + 1] * norm[3] + norm[2];
}

// Fallback policy for query s (rows [s0, s0+n) of the batch): a query whose e-value was
// computed (status & 1) from fewer than `sparse_below` candidates takes the learned line
// when it is usable (finite, falling); every other query keeps the plain fit.
__global__ void k_apply(gx_result *res, const float *pred, uint32_t s0, uint32_t n, uint32_t sparse_below,
                        double expect_max)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    gx_result r = res[s0 + i];
    if (!(r.status & 1) || (uint32_t)r.cpsms >= sparse_below) return;
    const double slope = (double)pred[2 * (size_t)i], lgs = (double)pred[2 * (size_t)i + 1];
    if (!isfinite(slope) || !isfinite(lgs) || !(slope < 0.0)) return;
    const double icpt = lgs - slope * (double)r.maxhyp;
    r.mu = to_int_x86(slope * 1e6);
    r.beta = to_int_x86(icpt * 1e6);
    const double w = (double)r.mu / 1e6, b = (double)r.beta / 1e6;
    r.e_x = pow(10.0, w * (double)r.maxhyp + b) * (double)(uint32_t)r.cpsms;
    r.status = (r.status & ~2) | GX_STATUS_LEARNED_TAIL | (r.e_x < expect_max ? 2 : 0);
    res[s0 + i] = r;
}

__global__ void k_all_queries(gx_tail_sample *smp, uint32_t s0, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) smp[i] = gx_tail_sample{s0 + i, 0u, 0ull};
}

inline unsigned blocks(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

}  // namespace tail
}  // namespace gx

using namespace gx;
using namespace gx::tail;

// ------------------------------------------------------------------------------------
// model object
// ------------------------------------------------------------------------------------
struct gx_tail_model {
    int device = 0;
    uint32_t max_batch = 0;
    uint64_t step = 0;
    float norm_h[4] = {0.f, 1.f, 0.f, 1.f};
    float huber = 0.0f;   // training loss: 0 squared error, > 0 Huber's loss with this delta
    float *P = nullptr, *G = nullptr, *m1 = nullptr, *m2 = nullptr, *norm = nullptr;
    bf16 *Pb = nullptr;
    float *Z1 = nullptr, *Z2 = nullptr, *Y = nullptr, *loss = nullptr, *pred = nullptr;
    bf16 *A1 = nullptr, *A2 = nullptr, *dY = nullptr, *dZ1 = nullptr, *dZ2 = nullptr, *X = nullptr;
    gx_tail_sample *smp = nullptr;
    int32_t *err = nullptr;
    std::vector<void *> allocs;
};

namespace {

std::mutex g_attr_mu;
bool g_attr_done[64] = {};
// limit of each tensor-core wait of k_gemm (gx_tail_set_wait_limit)
constexpr uint64_t kDefaultWaitNs = 1000000000ull;
std::atomic<uint64_t> g_wait_ns{kDefaultWaitNs};


gx_status set_attributes(int device)
{
    std::lock_guard<std::mutex> g(g_attr_mu);
    if (device < 0 || device >= 64) return fail(GX_ERR_INVLD_PARAM, "tail model: device id");
    if (g_attr_done[device]) return GX_SUCCESS;
    cudaError_t e = cudaFuncSetAttribute(k_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
    if (e != cudaSuccess) return cuda_fail(e, "tail model: k_gemm attributes");
    g_attr_done[device] = true;
    return GX_SUCCESS;
}

template <class T>
gx_status dalloc(gx_tail_model *m, T **p, size_t count)
{
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 16);
    if (e != cudaSuccess) return cuda_fail(e, "tail model: cudaMalloc");
    m->allocs.push_back(q);
    *p = static_cast<T *>(q);
    return GX_SUCCESS;
}

int ntile(int N)
{
    const int r = (N + 15) / 16 * 16;
    return r > 256 ? 256 : r;
}

gx_status gemm(const gx_tail_model *m, const bf16 *A, long long sam, long long sak, const bf16 *B, long long sbn,
               long long sbk, int M, int N, int K, int epi, float *D, long long ldd, bf16 *H, long long ldh,
               const float *bias, const float *Z, long long ldz, cudaStream_t st)
{
    if (M <= 0 || N <= 0 || K <= 0) return fail(GX_ERR_INVLD_SIZE, "tail model: empty GEMM");
    GemmArgs a{A,   sam, sak, B,    sbn, sbk, M, N, K, ntile(N), epi, D, ldd, H, ldh, bias, Z, ldz,
               m ? m->err : nullptr, g_wait_ns.load(std::memory_order_relaxed)};
    dim3 grid((unsigned)((M + 127) / 128), (unsigned)((N + a.NT - 1) / a.NT));
    int h = prof_begin("k_gemm", st);
    k_gemm<<<grid, kGemmThreads, kGemmSmem, st>>>(a);
    prof_end(h, st);
    count_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GX_SUCCESS : cuda_fail(e, "tail model: k_gemm launch");
}

#define GX_TRY(x)                                  \
    do {                                           \
        gx_status _s = (x);                        \
        if (_s != GX_SUCCESS) return _s;           \
    } while (0)

gx_status launched(const char *what)
{
    cudaError_t e = cudaGetLastError();
    count_launch();
    return e == cudaSuccess ? GX_SUCCESS : cuda_fail(e, what);
}

// forward pass over n rows of X (bf16 [n][kIn]) -> m->Y [n][2]
gx_status forward(gx_tail_model *m, const bf16 *X, uint32_t n, cudaStream_t st)
{
    const bf16 *W1 = m->Pb + kW1, *W2 = m->Pb + kW2, *W3 = m->Pb + kW3;
    GX_TRY(gemm(m, X, kIn, 1, W1, kIn, 1, (int)n, kHid, kIn, kEpiBiasGelu, m->Z1, kHid, m->A1, kHid, m->P + kB1,
                nullptr, 0, st));
    GX_TRY(gemm(m, m->A1, kHid, 1, W2, kHid, 1, (int)n, kHid, kHid, kEpiBiasGelu, m->Z2, kHid, m->A2, kHid,
                m->P + kB2, nullptr, 0, st));
    return gemm(m, m->A2, kHid, 1, W3, kHid, 1, (int)n, kOut, kHid, kEpiBias, m->Y, kOut, nullptr, 0, m->P + kB3,
                nullptr, 0, st);
}

// forward + loss + backward: gradients into m->G, mean loss added to m->loss
gx_status grads(gx_tail_model *m, const bf16 *X, const float *T, uint32_t n, float w0, float w1, cudaStream_t st)
{
    GX_TRY(forward(m, X, n, st));
    int h = prof_begin("k_loss", st);
    k_loss<<<blocks(n, 256), 256, 0, st>>>(m->Y, T, n, m->norm, w0, w1, m->huber, m->dY, m->loss);
    prof_end(h, st);
    GX_TRY(launched("tail model: k_loss"));
    float *G = m->G;
    const bf16 *W2 = m->Pb + kW2, *W3 = m->Pb + kW3;
    // layer 3: dW3 = dY^T A2, db3 = colsum dY, dZ2 = (dY W3) * GELU'(Z2)
    GX_TRY(gemm(m, m->dY, 1, kOut, m->A2, 1, kHid, kOut, kHid, (int)n, kEpiF32, G + kW3, kHid, nullptr, 0, nullptr,
                nullptr, 0, st));
    k_colsum<<<1, 32, 0, st>>>(m->dY, kOut, n, kOut, G + kB3);
    GX_TRY(launched("tail model: k_colsum"));
    GX_TRY(gemm(m, m->dY, kOut, 1, W3, 1, kHid, (int)n, kHid, kOut, kEpiDGelu, nullptr, 0, m->dZ2, kHid, nullptr,
                m->Z2, kHid, st));
    // layer 2
    GX_TRY(gemm(m, m->dZ2, 1, kHid, m->A1, 1, kHid, kHid, kHid, (int)n, kEpiF32, G + kW2, kHid, nullptr, 0, nullptr,
                nullptr, 0, st));
    k_colsum<<<blocks(kHid, 128), 128, 0, st>>>(m->dZ2, kHid, n, kHid, G + kB2);
    GX_TRY(launched("tail model: k_colsum"));
    GX_TRY(gemm(m, m->dZ2, kHid, 1, W2, 1, kHid, (int)n, kHid, kHid, kEpiDGelu, nullptr, 0, m->dZ1, kHid, nullptr,
                m->Z1, kHid, st));
    // layer 1
    GX_TRY(gemm(m, m->dZ1, 1, kHid, X, 1, kIn, kHid, kIn, (int)n, kEpiF32, G + kW1, kIn, nullptr, 0, nullptr,
                nullptr, 0, st));
    k_colsum<<<blocks(kHid, 128), 128, 0, st>>>(m->dZ1, kHid, n, kHid, G + kB1);
    return launched("tail model: k_colsum");
}

gx_status check_model(const gx_tail_model *m, uint32_t n, const char *what)
{
    if (!m) return fail(GX_ERR_INVLD_PTR, std::string(what) + ": null model");
    cudaGetLastError();   // an earlier call's error is not ours to report
    if (n > m->max_batch)
        return fail(GX_ERR_INVLD_SIZE, std::string(what) + ": batch of " + std::to_string(n) + " rows exceeds max_batch " +
                                           std::to_string(m->max_batch));
    return GX_SUCCESS;
}

// Checks the model and batch, then makes the model's device current for the rest of the
// calling entry point (the caller's device is current again when it returns).
#define GX_MODEL_SCOPE(m, n, what)                                              \
    GX_TRY(check_model(m, n, what));                                            \
    DeviceScope model_scope_((m)->device);                                      \
    if (model_scope_.status() != cudaSuccess) return cuda_fail(model_scope_.status(), what)

}  // namespace

// ------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------
extern "C" gx_status gx_tail_model_create(int32_t device, uint32_t max_batch, uint64_t seed, gx_tail_model **out)
{
    if (!out) return fail(GX_ERR_INVLD_PTR, "gx_tail_model_create: null out");
    cudaGetLastError();
    *out = nullptr;
    if (max_batch == 0 || max_batch > (1u << 22))
        return fail(GX_ERR_INVLD_SIZE, "gx_tail_model_create: max_batch must be in 1..2^22");
    DeviceScope ds(device);
    cudaError_t e = ds.status();
    if (e != cudaSuccess) return cuda_fail(e, "gx_tail_model_create: cudaSetDevice");
    GX_TRY(set_attributes(device));
    gx_tail_model *m = new gx_tail_model;
    m->device = device;
    m->max_batch = max_batch;
    const size_t B = max_batch;
    gx_status s = GX_SUCCESS;
    auto A = [&](auto **p, size_t cnt) {
        if (s == GX_SUCCESS) s = dalloc(m, p, cnt);
    };
    A(&m->P, kNParam); A(&m->G, kNParam); A(&m->m1, kNParam); A(&m->m2, kNParam); A(&m->norm, 4);
    A(&m->Pb, kNParam);
    A(&m->Z1, B * kHid); A(&m->Z2, B * kHid); A(&m->Y, B * kOut); A(&m->loss, 1); A(&m->pred, B * kOut);
    A(&m->A1, B * kHid); A(&m->A2, B * kHid); A(&m->dY, B * kOut); A(&m->dZ1, B * kHid); A(&m->dZ2, B * kHid);
    A(&m->X, B * kIn); A(&m->smp, B); A(&m->err, 1);
    if (s != GX_SUCCESS) {
        gx_tail_model_free(m);
        return s;
    }
    // initial weights: U(-1/sqrt(fan_in), 1/sqrt(fan_in)), biases zero
    std::vector<float> p(kNParam, 0.0f);
    std::mt19937_64 rng(seed);
    auto fill = [&](size_t off, int rows, int fan_in) {
        std::uniform_real_distribution<float> u(-1.0f / std::sqrt((float)fan_in), 1.0f / std::sqrt((float)fan_in));
        for (size_t i = 0; i < (size_t)rows * fan_in; i++) p[off + i] = u(rng);
    };
    fill(kW1, kHid, kIn);
    fill(kW2, kHid, kHid);
    fill(kW3, kOut, kHid);
    const float norm[4] = {0.f, 1.f, 0.f, 1.f};
    s = gx_tail_model_set(m, p.data(), norm);
    if (s == GX_SUCCESS && (e = cudaMemset(m->err, 0, sizeof(int32_t))) != cudaSuccess)
        s = cuda_fail(e, "gx_tail_model_create: cudaMemset");
    if (s != GX_SUCCESS) {
        gx_tail_model_free(m);
        return s;
    }
    *out = m;
    return GX_SUCCESS;
}

extern "C" gx_status gx_tail_model_free(gx_tail_model *m)
{
    if (!m) return GX_SUCCESS;
    DeviceScope ds(m->device);
    for (void *p : m->allocs) cudaFree(p);
    delete m;
    return GX_SUCCESS;
}

extern "C" gx_status gx_tail_model_set(gx_tail_model *m, const float *params, const float *norm)
{
    GX_MODEL_SCOPE(m, 0, "gx_tail_model_set");
    cudaError_t e;
    if (params) {
        if ((e = cudaMemcpy(m->P, params, kNParam * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
            return cuda_fail(e, "gx_tail_model_set: params");
        if ((e = cudaMemset(m->m1, 0, kNParam * sizeof(float))) != cudaSuccess ||
            (e = cudaMemset(m->m2, 0, kNParam * sizeof(float))) != cudaSuccess)
            return cuda_fail(e, "gx_tail_model_set: moments");
        m->step = 0;
        k_to_bf16<<<blocks(kNParam, 256), 256>>>(m->P, m->Pb, (uint32_t)kNParam);
        GX_TRY(launched("gx_tail_model_set: k_to_bf16"));
    }
    if (norm) {
        for (int i = 0; i < 4; i++) m->norm_h[i] = norm[i];
        if (!(norm[1] > 0.f) || !(norm[3] > 0.f))
            return fail(GX_ERR_INVLD_PARAM, "gx_tail_model_set: target scales must be > 0");
        if ((e = cudaMemcpy(m->norm, norm, 4 * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
            return cuda_fail(e, "gx_tail_model_set: norm");
    }
    e = cudaDeviceSynchronize();
    return e == cudaSuccess ? GX_SUCCESS : cuda_fail(e, "gx_tail_model_set");
}

extern "C" gx_status gx_tail_model_get(const gx_tail_model *m, float *params, float *norm, uint64_t *steps)
{
    GX_MODEL_SCOPE(m, 0, "gx_tail_model_get");
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "gx_tail_model_get");
    if (params && (e = cudaMemcpy(params, m->P, kNParam * sizeof(float), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "gx_tail_model_get: params");
    if (norm) for (int i = 0; i < 4; i++) norm[i] = m->norm_h[i];
    if (steps) *steps = m->step;
    return GX_SUCCESS;
}

extern "C" gx_status gx_tail_features(gx_tail_model *m, const uint32_t *hist_dev, const gx_result *res_dev,
                                      const float *prec_dev, const int32_t *charge_dev, uint32_t nq,
                                      const gx_tail_sample *samples_host, uint32_t n, uint16_t *x_dev,
                                      uint32_t *sub_hist_dev, int32_t *sub_cpsms_dev, int32_t *hyp_dev, void *stream)
{
    GX_MODEL_SCOPE(m, n, "gx_tail_features");
    if (n == 0) return GX_SUCCESS;
    if (!hist_dev || !res_dev || !prec_dev || !samples_host || !x_dev)
        return fail(GX_ERR_INVLD_PTR, "gx_tail_features: null argument");
    for (uint32_t i = 0; i < n; i++) {
        if (samples_host[i].query >= nq)
            return fail(GX_ERR_INVLD_PARAM, "gx_tail_features: sample " + std::to_string(i) + " names query " +
                                                std::to_string(samples_host[i].query) + " of " + std::to_string(nq));
        if (samples_host[i].keep > GX_TAIL_MAX_KEEP)
            return fail(GX_ERR_INVLD_PARAM, "gx_tail_features: keep above GX_TAIL_MAX_KEEP");
    }
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(m->smp, samples_host, n * sizeof(gx_tail_sample), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "gx_tail_features: samples");
    FeatArgs a{hist_dev, res_dev, prec_dev, charge_dev, m->smp, n, nq, reinterpret_cast<bf16 *>(x_dev),
               sub_hist_dev, sub_cpsms_dev, hyp_dev, m->err};
    int h = prof_begin("k_features", st);
    k_features<<<blocks(n, kFeatWarps), kFeatWarps * 32, 0, st>>>(a);
    prof_end(h, st);
    GX_TRY(launched("gx_tail_features: launch"));
    // the sample table is reused by the next call: keep the host copy alive until here
    e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? GX_SUCCESS : cuda_fail(e, "gx_tail_features");
}

extern "C" gx_status gx_tail_fit_rows(const uint32_t *hist_dev, const int32_t *cpsms_dev, const int32_t *hyp_dev,
                                      uint32_t n, double *fit_dev, void *stream)
{
    if (n == 0) return GX_SUCCESS;
    if (!hist_dev || !cpsms_dev || !hyp_dev || !fit_dev) return fail(GX_ERR_INVLD_PTR, "gx_tail_fit_rows: null argument");
    cudaGetLastError();
    cudaStream_t st = (cudaStream_t)stream;
    int h = prof_begin("k_fit_rows", st);
    k_fit_rows<<<blocks(n, kFitWarps), kFitWarps * 32, 0, st>>>(hist_dev, cpsms_dev, hyp_dev, n, fit_dev);
    prof_end(h, st);
    return launched("gx_tail_fit_rows: launch");
}

extern "C" gx_status gx_tail_grad(gx_tail_model *m, const uint16_t *x_dev, const float *target_dev, uint32_t n,
                                  const float *weights2, float *grad_dev, float *loss_dev, void *stream)
{
    GX_MODEL_SCOPE(m, n, "gx_tail_grad");
    if (n == 0 || !x_dev || !target_dev) return fail(GX_ERR_INVLD_PARAM, "gx_tail_grad: empty batch or null input");
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(m->loss, 0, sizeof(float), st);
    if (e != cudaSuccess) return cuda_fail(e, "gx_tail_grad: loss");
    const float w0 = weights2 ? weights2[0] : 1.0f, w1 = weights2 ? weights2[1] : 1.0f;
    GX_TRY(grads(m, reinterpret_cast<const bf16 *>(x_dev), target_dev, n, w0, w1, st));
    if (grad_dev && (e = cudaMemcpyAsync(grad_dev, m->G, kNParam * sizeof(float), cudaMemcpyDeviceToDevice, st)) !=
                        cudaSuccess)
        return cuda_fail(e, "gx_tail_grad: copy gradients");
    if (loss_dev && (e = cudaMemcpyAsync(loss_dev, m->loss, sizeof(float), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "gx_tail_grad: copy loss");
    return GX_SUCCESS;
}

extern "C" gx_status gx_tail_train_step(gx_tail_model *m, const uint16_t *x_dev, const float *target_dev, uint32_t n,
                                        const gx_tail_adam *opt, float *loss_dev, void *stream)
{
    GX_MODEL_SCOPE(m, n, "gx_tail_train_step");
    if (n == 0 || !x_dev || !target_dev || !opt)
        return fail(GX_ERR_INVLD_PARAM, "gx_tail_train_step: empty batch or null input");
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(m->loss, 0, sizeof(float), st);
    if (e != cudaSuccess) return cuda_fail(e, "gx_tail_train_step: loss");
    GX_TRY(grads(m, reinterpret_cast<const bf16 *>(x_dev), target_dev, n, opt->w_slope, opt->w_lgs, st));
    m->step++;
    const float bc1 = 1.0f - (float)std::pow((double)opt->beta1, (double)m->step);
    const float bc2 = 1.0f - (float)std::pow((double)opt->beta2, (double)m->step);
    int h = prof_begin("k_adam", st);
    k_adam<<<blocks(kNParam, 256), 256, 0, st>>>(m->P, m->G, m->m1, m->m2, m->Pb, (uint32_t)kNParam, opt->lr,
                                                 opt->beta1, opt->beta2, opt->eps, bc1, bc2);
    prof_end(h, st);
    GX_TRY(launched("gx_tail_train_step: k_adam"));
    if (loss_dev && (e = cudaMemcpyAsync(loss_dev, m->loss, sizeof(float), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "gx_tail_train_step: copy loss");
    return GX_SUCCESS;
}

extern "C" gx_status gx_tail_predict(gx_tail_model *m, const uint16_t *x_dev, uint32_t n, float *pred_dev, void *stream)
{
    GX_MODEL_SCOPE(m, n, "gx_tail_predict");
    if (n == 0) return GX_SUCCESS;
    if (!x_dev || !pred_dev) return fail(GX_ERR_INVLD_PTR, "gx_tail_predict: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    GX_TRY(forward(m, reinterpret_cast<const bf16 *>(x_dev), n, st));
    k_predict<<<blocks(n, 256), 256, 0, st>>>(m->Y, n, m->norm, pred_dev);
    return launched("gx_tail_predict: k_predict");
}

extern "C" gx_status gx_tail_apply(gx_tail_model *m, const uint32_t *hist_dev, gx_result *res_dev,
                                   const float *prec_dev, const int32_t *charge_dev, uint32_t nspec,
                                   uint32_t sparse_below, double expect_max, void *stream)
{
    GX_MODEL_SCOPE(m, 0, "gx_tail_apply");
    if (nspec == 0 || sparse_below == 0) return GX_SUCCESS;
    if (!hist_dev || !res_dev || !prec_dev) return fail(GX_ERR_INVLD_PTR, "gx_tail_apply: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    for (uint32_t s0 = 0; s0 < nspec; s0 += m->max_batch) {
        const uint32_t n = std::min(m->max_batch, nspec - s0);
        k_all_queries<<<blocks(n, 256), 256, 0, st>>>(m->smp, s0, n);
        GX_TRY(launched("gx_tail_apply: samples"));
        FeatArgs a{hist_dev, res_dev, prec_dev, charge_dev, m->smp, n, nspec, m->X, nullptr, nullptr, nullptr, m->err};
        int h = prof_begin("k_features", st);
        k_features<<<blocks(n, kFeatWarps), kFeatWarps * 32, 0, st>>>(a);
        prof_end(h, st);
        GX_TRY(launched("gx_tail_apply: k_features"));
        GX_TRY(forward(m, m->X, n, st));
        k_predict<<<blocks(n, 256), 256, 0, st>>>(m->Y, n, m->norm, m->pred);
        GX_TRY(launched("gx_tail_apply: k_predict"));
        h = prof_begin("k_apply", st);
        k_apply<<<blocks(n, 256), 256, 0, st>>>(res_dev, m->pred, s0, n, sparse_below, expect_max);
        prof_end(h, st);
        GX_TRY(launched("gx_tail_apply: k_apply"));
    }
    return GX_SUCCESS;
}

extern "C" gx_status gx_tail_check(gx_tail_model *m)
{
    GX_MODEL_SCOPE(m, 0, "gx_tail_check");
    int32_t v = 0;
    cudaError_t e = cudaMemcpy(&v, m->err, sizeof(v), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "gx_tail_check");
    if (v == 0) return GX_SUCCESS;
    if ((e = cudaMemset(m->err, 0, sizeof(int32_t))) != cudaSuccess) return cuda_fail(e, "gx_tail_check: clear");
    if (v == 1) return fail(GX_ERR_DEVICE_GUARD, "tail model: a sample had an invalid top bin");
    return fail(GX_ERR_DEVICE_GUARD, "tail model: a tensor-core wait ran out");
}

extern "C" gx_status gx_tail_set_loss(gx_tail_model *m, float huber_delta)
{
    if (!m) return fail(GX_ERR_INVLD_PTR, "gx_tail_set_loss: null model");
    if (!(huber_delta >= 0.0f) || !std::isfinite(huber_delta))
        return fail(GX_ERR_INVLD_PARAM, "gx_tail_set_loss: the Huber delta must be finite and >= 0");
    m->huber = huber_delta;
    return GX_SUCCESS;
}

extern "C" gx_status gx_tail_set_wait_limit(uint64_t ns)
{
    g_wait_ns.store(ns, std::memory_order_relaxed);
    return GX_SUCCESS;
}

extern "C" gx_status gx_tail_gemm(const uint16_t *a_dev, int64_t sam, int64_t sak, const uint16_t *b_dev, int64_t sbn,
                                  int64_t sbk, int32_t M, int32_t N, int32_t K, float *d_dev, int64_t ldd, void *stream)
{
    if (!a_dev || !b_dev || !d_dev) return fail(GX_ERR_INVLD_PTR, "gx_tail_gemm: null argument");
    cudaGetLastError();
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "gx_tail_gemm: cudaGetDevice");
    GX_TRY(set_attributes(dev));
    return gemm(nullptr, reinterpret_cast<const bf16 *>(a_dev), sam, sak, reinterpret_cast<const bf16 *>(b_dev), sbn,
                sbk, M, N, K, kEpiF32, d_dev, ldd, nullptr, 0, nullptr, nullptr, 0, (cudaStream_t)stream);
}
