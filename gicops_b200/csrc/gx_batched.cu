// Batched query path: one persistent kernel fed by a work queue of spectra sorted by
// their scan volume, heaviest first.
//
//   k_prep          per spectrum: precursor windows of every length, the peak windows
//                   merged into disjoint bin intervals (coverage count, intensity sum),
//                   the packed-scorecard guard and the scan volume (sort key)
//   (radix sort of the spectra by scan volume, descending)
//   k_search_batched  persistent CTAs (two per SM); per spectrum, per length, per
//                   candidate tile (one block of the block layout): stream the 16-bit ids
//                   of every interval (each bucket read once) into the BYC scorecard in
//                   shared memory, then scan the tile in entry order (hyperscore,
//                   histogram, exact top-K heap)
//   k_search_piped  (launch-shape option) one CTA of 32 warps per SM with two scorecard
//                   tiles: tile t scored while tile t + 1 streams, one barrier per tile; it
//                   takes the 8-byte-scorecard spectra of at most 256 intervals and
//                   k_search_batched the others
//   k_tailfit       one warp per spectrum: expeRT tail fit and e-value
//
// Results are identical to the reference's CPU path (source/core/dslim_query.cpp:
// 827-1061): every (peak, bin, ion) match of the reference is counted once per
// covering peak, through the interval's coverage count and intensity sum.

#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include "../../include/gicops_b200.h"
#include "gx_batched.h"
#include "gx_device.cuh"
#include "gx_index.cuh"
#include "gx_internal.h"

namespace gx {

// ------------------------------------------------------------------------------------
// k_prep: one CTA per spectrum
// ------------------------------------------------------------------------------------
constexpr int kPrepBlock = 256;
// guard word of a spectrum k_prep rejects (more than GX_MAX_PEAKS peaks, or more intervals
// than the workspace holds); 0 and 1 say whether the packed scorecard is exact
constexpr uint32_t kGuardRejected = 2u;

__global__ void __launch_bounds__(kPrepBlock) k_prep(SearchArgs a, int2 *win, uint64_t *work_key, uint32_t *order0)
{
    __shared__ int32_t pk[GX_MAX_PEAKS];
    __shared__ uint32_t pi[GX_MAX_PEAKS];
    __shared__ int32_t npk_s;
    __shared__ unsigned long long red[kPrepBlock / 32];
    __shared__ uint32_t nv_s;
    __shared__ int2 win_s[GX_MAX_LENGTHS];
    const int tid = threadIdx.x;
    const uint32_t s = blockIdx.x;
    if (s >= a.nspec) return;
    const uint32_t q0 = a.qidx[s], q1 = a.qidx[s + 1];
    if (tid == 0) npk_s = 0;
    __syncthreads();
    if (q1 < q0 || q1 - q0 > GX_MAX_PEAKS || 2ull * q1 > a.ivl_cap) {
        if (tid == 0) {
            atomicExch(a.err, 1);
            a.nivl[s] = 0;
            a.guard[s] = kGuardRejected;   // k_search_batched writes the spectrum's flagged empty row
            work_key[s] = 0;
            order0[s] = s;
        }
        for (int l = tid; l < a.nlen; l += kPrepBlock) win[(uint64_t)s * a.nlen + l] = make_int2(1, 0);
        return;
    }
    // valid peaks (those the reference probes), padded to a power of two for the sort
    unsigned long long isum = 0;
    for (uint32_t k = q0 + tid; k < q1; k += kPrepBlock) {
        const int32_t m = a.moz[k];
        if (m > (int32_t)a.dF && (double)m < a.upper) {
            const int slot = atomicAdd(&npk_s, 1);
            pk[slot] = m;
            pi[slot] = (uint32_t)a.intn[k];
            isum += (uint32_t)a.intn[k];
        }
    }
    __syncthreads();
    const int n = npk_s;
    int np2 = 1;
    while (np2 < n) np2 <<= 1;
    for (int i = n + tid; i < np2; i += kPrepBlock) {
        pk[i] = 0x7fffffff;
        pi[i] = 0;
    }
    __syncthreads();
    // bitonic sort of (m/z, intensity) by m/z
    for (int k = 2; k <= np2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < np2; i += kPrepBlock) {
                const int l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    if ((pk[i] > pk[l]) == up) {
                        const int32_t t = pk[i]; pk[i] = pk[l]; pk[l] = t;
                        const uint32_t u = pi[i]; pi[i] = pi[l]; pi[l] = u;
                    }
                }
            }
            __syncthreads();
        }
    // guard of the packed scorecard: counts < 256 and sums < 2^24 per candidate
    for (int o = 16; o; o >>= 1) isum += __shfl_xor_sync(0xffffffffu, isum, o);
    if ((tid & 31) == 0) red[tid >> 5] = isum;
    __syncthreads();
    if (tid == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kPrepBlock / 32; w++) t += red[w];
        a.guard[s] = ((uint64_t)n * a.maxz <= 255u && t * a.maxz < (1ull << 24)) ? 1u : 0u;
        // sweep: windows [m-dF, m+dF] of sorted peaks start and end in the same order
        Interval *out = a.ivl + 2ull * q0;
        uint32_t nv = 0, c = 0, S = 0;
        int is = 0, ie = 0;
        int64_t prev = 0;
        const int64_t dF = a.dF;
        while (ie < n) {
            const int64_t ps = is < n ? (int64_t)pk[is] - dF : INT64_MAX;
            const int64_t pe = (int64_t)pk[ie] + dF + 1;
            const int64_t pos = ps < pe ? ps : pe;
            if (c > 0) out[nv++] = Interval{(uint32_t)prev, (uint32_t)(pos - 1), c, S};
            while (ie < n && (int64_t)pk[ie] + dF + 1 == pos) { c--; S -= pi[ie]; ie++; }
            while (is < n && (int64_t)pk[is] - dF == pos) { c++; S += pi[is]; is++; }
            prev = pos;
        }
        a.nivl[s] = nv;
        nv_s = nv;
    }
    __syncthreads();
    // windows and scan volume
    const double dM = a.dMq ? a.dMq[s] : a.dM;
    const float pr = a.prec[s];
    const float p1 = __double2float_rn(__dsub_rn((double)pr, dM));
    const float p2 = __double2float_rn(__dadd_rn((double)pr, dM));
    unsigned long long vol = 0;
    const uint32_t nv = nv_s;
    const Interval *iv = a.ivl + 2ull * q0;
    // thread l: the window of length l (the binary searches of all lengths run side by side)
    if (tid < a.nlen) {
        const DevLen ln = a.lens[tid];
        int lo = 1, hi = 0;
        if (!(dM < 0.0) && ln.npep > 0) {
            const float *m = a.mass + ln.mass_off;
            const uint32_t N = ln.npep;
            if (p1 == p1 && p2 == p2 && !(p1 > m[N - 1]) && !(p2 < m[0])) {
                uint32_t x = 0, y = N;
                while (x < y) { const uint32_t c = (x + y) >> 1; if (m[c] < p1) x = c + 1; else y = c; }
                lo = (int)x;
                x = 0; y = N;
                while (x < y) { const uint32_t c = (x + y) >> 1; if (p2 < m[c]) y = c; else x = c + 1; }
                hi = (int)x - 1;
            }
        }
        win_s[tid] = make_int2(lo, hi);
        win[(uint64_t)s * a.nlen + tid] = make_int2(lo, hi);
    }
    __syncthreads();
    // scan volume: ids of every (interval, length) pair with a window, times its tiles
    const uint32_t npair = nv * (uint32_t)a.nlen;
#pragma unroll 4
    for (uint32_t pq = tid; pq < npair; pq += kPrepBlock) {
        const uint32_t l = pq / nv, i = pq - l * nv;
        const int2 wv = win_s[l];
        if (wv.y >= wv.x) {
            const uint32_t W = (uint32_t)(wv.y - wv.x + 1);
            const uint32_t ntiles = (W + (uint32_t)a.tile - 1) / (uint32_t)a.tile;
            const uint32_t *bA = a.bA + (uint64_t)l * a.nbins;
            vol += (unsigned long long)(__ldg(bA + iv[i].b1 + 1) - __ldg(bA + iv[i].b0)) * ntiles;
        }
    }
    if (tid < a.nlen && win_s[tid].y >= win_s[tid].x) vol += (uint32_t)(win_s[tid].y - win_s[tid].x + 1);
    for (int o = 16; o; o >>= 1) vol += __shfl_xor_sync(0xffffffffu, vol, o);
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = vol;
    __syncthreads();
    if (tid == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kPrepBlock / 32; w++) t += red[w];
        work_key[s] = t;
        order0[s] = s;
    }
}

// ------------------------------------------------------------------------------------
// k_search_batched
// ------------------------------------------------------------------------------------
#ifndef GX_BATCH_WARPS
#define GX_BATCH_WARPS 16
#endif
constexpr int kBWarps = GX_BATCH_WARPS;      // warps per CTA
constexpr int kBBlock = kBWarps * 32;
#ifndef GX_CTAS_PER_SM
#define GX_CTAS_PER_SM (1024 / (GX_BATCH_WARPS * 32))
#endif
constexpr int kCtasPerSm = GX_CTAS_PER_SM;   // resident CTAs per SM (each its own spectrum)
#ifndef GX_PEND
#define GX_PEND 160
#endif
constexpr int kPend = GX_PEND;  // per-warp queue of candidates awaiting a hyperscore (32 + one scan step)
static_assert(kPend >= 128, "the queue must hold one scan step's candidates (32 lanes x 4)");
constexpr int kIvlChunk = 256;  // intervals per span table
constexpr int kDummy = 32;      // scorecard words that take the adds of ids outside the tile (one per lane)
// 16-byte id chunks each lane loads per work unit before it scatters any: a template
// parameter of the kernel (1..kMaxChunks), chosen per launch (BatchedTiles::chunks)
constexpr int kMaxChunks = 3;
// The last warp inserts heap entrants while the others stream, and builds the next tile's
// span table while the others scan and score (it takes no share of the scan).
constexpr int kHeapWarp = kBWarps - 1;
constexpr int kScanWarps = kBWarps - 1;
constexpr int kUnitTab = 64;   // stream units whose first interval the warp-built span table records
// Candidates of a tile of tn that each scanning warp owns (a multiple of the scan step): at
// most the length of the warp's entrant list.
__host__ __device__ constexpr int scan_range(int tn, int step)
{
    return ((tn + kScanWarps - 1) / kScanWarps + step - 1) / step * step;
}
#ifndef GX_ENT_SMEM
#define GX_ENT_SMEM 8
#endif
constexpr int kEntSmem = GX_ENT_SMEM;   // heap entrants per warp kept in shared memory
#ifndef GX_WARP_SEARCH
#define GX_WARP_SEARCH 1   // a unit's first interval found by a two-level warp search (0: binary search)
#endif
static_assert(kIvlChunk <= 256, "the warp search covers 32 x 8 span-table entries");
#ifndef GX_STREAM_PREFETCH
#define GX_STREAM_PREFETCH 0   // stream: the next unit's chunks loaded before the current one's are scattered
#endif
#ifndef GX_FUSED_CLEAR
#define GX_FUSED_CLEAR 1   // packed scorecard reset during the scan and after scoring (0: one pass after)
#endif


// Dynamic shared memory after the scorecard tile (tile * 8 bytes):
//   dummy      kDummy words right after the scorecard, written and never read
//   pend       per-warp queue of candidate offsets awaiting a hyperscore
//   span table of up to kIvlChunk intervals, in the current block of the current length
//              (element indices relative to the length's 16-byte aligned base), one
//              16-byte record per interval: x = q0 - pre (q0 = 16-byte chunk of the first
//              id, so that chunk j of the table is x + j), [y, z) = the interval's ids,
//              w = the add of one id (packed: c << 24 | S; wide: S), with c, S the
//              coverage count and intensity sum; sp_c = c (wide scorecard); pre =
//              exclusive prefix of the intervals' chunk counts (kIvlChunk + 1)
struct BatchDyn {
    uint32_t (*pend)[kPend];
    uint4 *sp_rec;
    uint32_t *sp_c, *sp_pre;
    uint32_t *nx_s, *nx_e;   // block offsets of the next tile's intervals
};

__host__ __device__ constexpr size_t batch_dyn_bytes(int)
{
    return sizeof(uint32_t) * ((size_t)kDummy + (size_t)kBWarps * kPend + 7 * (size_t)kIvlChunk + (kIvlChunk + 4));
}

__device__ __forceinline__ BatchDyn carve_dyn(unsigned char *base)
{
    BatchDyn d;
    uint32_t *p = reinterpret_cast<uint32_t *>(base) + kDummy;
    d.pend = reinterpret_cast<uint32_t (*)[kPend]>(p);
    p += kBWarps * kPend;
    d.sp_rec = reinterpret_cast<uint4 *>(p); p += 4 * kIvlChunk;   // 16-byte aligned (see batch_dyn_bytes)
    d.sp_c = p; p += kIvlChunk;
    d.nx_s = p; p += kIvlChunk;
    d.nx_e = p; p += kIvlChunk;
    d.sp_pre = p;
    return d;
}

struct BatchSmem {
    uint32_t hist[kHist];
    double lgf[81];
    Cell heap[kMaxHeap + 1];

    uint32_t scan_tmp[kBWarps];
    int32_t warp_cnt[kBWarps];
    Cell ent_s[kBWarps][kEntSmem];   // first heap entrants of each warp (the rest spill to global)
    int32_t heap_size;
    int32_t cpsms;
    int32_t status;
    int32_t spec;
    uint32_t next_unit;
    uint32_t ent_mask;               // warps with entrants in the last scored tile
    uint32_t ready;                  // the span table of the next tile is built
    uint32_t unit_n;                 // stream units whose first interval unit_k holds (0: none)
    float root;
    // keep masks of a 16-byte chunk's eight ids: keep_lo[m] keeps ids m.., keep_hi[m]
    // keeps ids ..m (index m - 1)
    uint4 keep_lo[8];
    uint4 keep_hi[8];
    uint8_t unit_k[kUnitTab];        // interval of the first chunk of each of the first stream units
};

// Block-local ids are 2*(entry - block start) + (y ion); the tile's ids satisfy
// id - lo < lim.  Packed scorecard: per candidate a b word and a y word (count << 24 |
// intensity sum), interleaved, so that id - lo is the word an id adds to; 32-bit adds
// whose old values are not needed.
// Ids outside the tile (or, with ok false, outside the interval) add to the lane's dummy word.
__device__ __forceinline__ void scatter_packed(uint32_t *sc, uint32_t id, uint32_t lo, uint32_t lim, uint32_t vb,
                                               uint32_t dummy, bool ok)
{
    const uint32_t rel = id - lo;
    atomicAdd(sc + ((rel < lim && ok) ? rel : dummy), vb);
}

// Wide scorecard (12 bytes): counts b | y << 16, intensity sums of b and y ions.
__device__ __forceinline__ void scatter_wide(uint32_t *cnt, uint32_t *ib, uint32_t *iy, uint32_t id, uint32_t lo,
                                             uint32_t lim, uint32_t c, uint32_t S)
{
    const uint32_t rel = id - lo;
    if (rel < lim) {
        const uint32_t cand = rel >> 1;
        const bool y = rel & 1u;
        atomicAdd(cnt + cand, y ? (c << 16) : c);
        atomicAdd((y ? iy : ib) + cand, S);
    }
}

// Hyperscores of the n <= kPend queued candidates of a warp, in queue order: the
// histogram and candidate count take every PSM; PSMs with h >= tau go, in order, to the
// warp's entrant list for the exact heap.  Per 64 candidates, all scorecard reads and
// log10 table loads are issued before any hyperscore is formed.
template <class SM, int ENT_SMEM>
__device__ __forceinline__ void score_batch(SM &sm, const uint32_t *pend, const SearchArgs &a, const void *scv,
                                            int ctile, int wid, int lane, int n, int t0, int ixx, uint32_t speclen,
                                            float tau, bool wide, Cell *ent, int &nent, int &cps)
{
    constexpr int kG = 2;
    for (int q0 = 0; q0 < n; q0 += 32 * kG) {
    uint32_t off[kG], bc[kG], yc[kG], ib[kG], iy[kG];
    double lb[kG], ly[kG];
#pragma unroll
    for (int g = 0; g < kG; g++) {
        off[g] = 0; bc[g] = yc[g] = ib[g] = iy[g] = 0;
        if (q0 + 32 * g + lane < n) {
            off[g] = pend[q0 + 32 * g + lane];
            if (!wide) {
                const uint2 v = reinterpret_cast<const uint2 *>(scv)[off[g]];
                bc[g] = v.x >> 24; ib[g] = v.x & 0xFFFFFFu; yc[g] = v.y >> 24; iy[g] = v.y & 0xFFFFFFu;
            } else {
                const uint32_t *cnt = reinterpret_cast<const uint32_t *>(scv);
                const uint32_t cv = cnt[off[g]];
                bc[g] = cv & 0xFFFFu; yc[g] = cv >> 16;
                ib[g] = cnt[ctile + off[g]]; iy[g] = cnt[2 * ctile + off[g]];
            }
        }
    }
#pragma unroll
    for (int g = 0; g < kG; g++) {
        // log10 of small integers from a table filled by the same log10 (identical values)
        const uint32_t xb = 1u + ib[g], xy = 1u + iy[g];
        lb[g] = xb < a.logtab_n ? __ldg(a.logtab + xb) : log10((double)xb);
        ly[g] = xy < a.logtab_n ? __ldg(a.logtab + xy) : log10((double)xy);
    }
#pragma unroll
    for (int g = 0; g < kG; g++) {
        if (q0 + 32 * g >= n) break;
        bool psm = false;
        Cell cell;
        if (q0 + 32 * g + lane < n) {
            uint32_t bi = bc[g], yi = yc[g];
            if (bi > 80u || yi > 80u) {
                atomicOr(&sm.status, 4);
                bi = min(bi, 80u);
                yi = min(yi, 80u);
            }
            const double h1 = sm.lgf[bi] + sm.lgf[yi];
            float h = __double2float_rn(h1 + lb[g] + ly[g] - 4.0);
            if (h > 0.0f) {
                if (h >= 80.0f) h = 79.0f;
                psm = true;
                cell.h = h;
                cell.psid = t0 + (int)off[g];
                cell.ixx = (uint16_t)ixx;
                cell.shp = (uint16_t)((bc[g] + yc[g]) & 0xFFFFu);
                cell.total = (uint16_t)speclen;
                cell.pad = 0;
                const int hb = __double2int_rz(__dadd_rn((double)__fmul_rn(h, 10.0f), 0.5));
                atomicAdd(&sm.hist[hb], 1u);
            }
        }
        const unsigned pb = __ballot_sync(0xffffffffu, psm);
        cps += __popc(pb);
        const bool e = psm && cell.h >= tau;
        const unsigned eb = __ballot_sync(0xffffffffu, e);
        if (e) {
            const int gi = nent + __popc(eb & ((1u << lane) - 1u));
            if constexpr (ENT_SMEM > 0) {
                if (gi < ENT_SMEM) sm.ent_s[wid][gi] = cell;
                else ent[gi] = cell;
            } else {
                ent[gi] = cell;
            }
        }
        nent += __popc(eb);
    }
    }
}

// Resets the packed-scorecard groups (four candidates, 32 bytes) of the n scored
// candidates in q: the scan left every group holding a PSM as it was, for the scoring.
__device__ __forceinline__ void clear_scored(uint32_t *sw, const uint32_t *q, int n, int lane)
{
    for (int i = lane; i < n; i += 32) {
        uint4 *z = reinterpret_cast<uint4 *>(sw + 2 * (q[i] & ~3u));
        z[0] = make_uint4(0u, 0u, 0u, 0u);
        z[1] = make_uint4(0u, 0u, 0u, 0u);
    }
}

// Warp kHeapWarp inserts the entrants of the warps that have some (in warp order) of the
// last scored tile into the heap, in the order a single thread would: the first few of
// each warp from shared memory, any overflow from the warp's global spill.  The warp loads
// 32 entrants at a time (the next 32 in flight while these are inserted); once the heap is
// full, a cell below its root is rejected by heap_insert and the root never decreases, so
// the lanes drop the cells below the root at the start of the batch and lane 0 inserts
// only the others.  Every lane tracks the heap size (an insertion into a heap that is not
// full always appends).
__device__ __noinline__ void insert_entrants(BatchSmem &sm, const Cell *spill_cta, uint32_t spill_per_warp, int cap,
                                             int lane)
{
    int hs = sm.heap_size;
    const uint32_t mask0 = sm.ent_mask;
    for (uint32_t mask = mask0; mask; mask &= mask - 1u) {
        const int w2 = __ffs(mask) - 1;
        const int n2 = sm.warp_cnt[w2];
        const Cell *e2 = spill_cta + (uint64_t)w2 * spill_per_warp;
        Cell nxt;
        if (lane < n2) nxt = lane < kEntSmem ? sm.ent_s[w2][lane] : e2[lane];
        for (int k0 = 0; k0 < n2; k0 += 32) {
            const Cell c = nxt;
            const bool v = k0 + lane < n2;
            const int k1 = k0 + 32 + lane;
            if (k1 < n2) nxt = e2[k1];
            __syncwarp();
            const float root = hs == cap ? sm.heap[0].h : -INFINITY;
            uint32_t live = __ballot_sync(0xffffffffu, v && c.h >= root);
            const uint32_t u1 = ((uint32_t)c.ixx) | ((uint32_t)c.shp << 16);
            const uint32_t u2 = ((uint32_t)c.total) | ((uint32_t)c.pad << 16);
            while (live) {
                const int j = __ffs(live) - 1;
                live &= live - 1u;
                Cell cj;
                cj.h = __shfl_sync(0xffffffffu, c.h, j);
                cj.psid = __shfl_sync(0xffffffffu, c.psid, j);
                const uint32_t v1 = __shfl_sync(0xffffffffu, u1, j), v2 = __shfl_sync(0xffffffffu, u2, j);
                cj.ixx = (uint16_t)(v1 & 0xFFFFu); cj.shp = (uint16_t)(v1 >> 16);
                cj.total = (uint16_t)(v2 & 0xFFFFu); cj.pad = (uint16_t)(v2 >> 16);
                if (lane == 0) {
                    int h0 = hs;
                    heap_insert(sm.heap, h0, cap, cj);
                }
                hs = min(hs + 1, cap);
            }
        }
    }
    __syncwarp();
    if (lane == 0) {
        sm.heap_size = hs;
        sm.root = sm.heap[0].h;
        sm.ent_mask = 0u;
    }
}

// Span table of up to kIvlChunk intervals for one block of one length (element indices
// relative to the length's aligned base, which lies rel0 elements before its first id),
// and the exclusive prefix of the intervals' 16-byte chunk counts.  With `have`, thread i
// already holds the block offsets of interval i (loaded one tile ahead).
__device__ __forceinline__ void build_span_table(BatchSmem &sm, const BatchDyn &dd, const Interval *iv, uint32_t n,
                                                 const uint32_t *__restrict__ bA, uint32_t rel0, bool have,
                                                 uint32_t have_s, uint32_t have_e, bool wide, int tid, int lane,
                                                 int wid)
{
    uint32_t cnt = 0, rq0 = 0;
    if (tid < (int)n) {
        const Interval v = iv[tid];
        const uint32_t a0 = rel0 + (have ? have_s : __ldg(bA + v.b0));
        const uint32_t a1 = rel0 + (have ? have_e : __ldg(bA + v.b1 + 1));
        const uint32_t q0 = a0 >> 3;
        cnt = a1 > a0 ? ((a1 + 7u) >> 3) - q0 : 0u;
        rq0 = q0;
        dd.sp_rec[tid] = make_uint4(0u, a0, a1, wide ? v.S : ((v.c << 24) | v.S));
        dd.sp_c[tid] = v.c;
    }
    if (tid == 0) {
        sm.next_unit = 0;
        sm.unit_n = 0;   // the stream finds each unit's first interval by search
    }
    // block exclusive scan of cnt
    uint32_t x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sm.scan_tmp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = lane < kBWarps ? sm.scan_tmp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < kBWarps) sm.scan_tmp[lane] = t;
    }
    __syncthreads();
    const uint32_t incl = x + (wid ? sm.scan_tmp[wid - 1] : 0u);
    if (tid < (int)n) {
        dd.sp_pre[tid] = incl - cnt;
        dd.sp_rec[tid].x = rq0 - (incl - cnt);
    }
    if (tid == (int)n - 1) dd.sp_pre[n] = incl;
    if (n == 0 && tid == 0) dd.sp_pre[0] = 0;
}

// The span table of the next tile, built by one warp from the offsets in nx_s / nx_e
// while the other warps score (the adds of the spectrum's intervals, record field w and
// sp_c, stay in place); it also resets the unit counter and records the interval of the first
// chunk of each of the first kUnitTab stream units (units of 32 x CH chunks).
template <int CH>
__device__ __forceinline__ void build_span_warp(BatchSmem &sm, const BatchDyn &dd, uint32_t n, uint32_t rel0, int lane)
{
    constexpr int kPer = kIvlChunk / 32;
    const uint32_t i0 = (uint32_t)lane * kPer;
    uint32_t cnt[kPer], q0s[kPer];
    uint32_t sum = 0;
#pragma unroll
    for (int j = 0; j < kPer; j++) {
        const uint32_t i = i0 + j;
        cnt[j] = 0;
        q0s[j] = 0;
        if (i < n) {
            const uint32_t a0 = rel0 + dd.nx_s[i], a1 = rel0 + dd.nx_e[i];
            const uint32_t q0 = a0 >> 3;
            cnt[j] = a1 > a0 ? ((a1 + 7u) >> 3) - q0 : 0u;
            q0s[j] = q0;
            dd.sp_rec[i].y = a0;
            dd.sp_rec[i].z = a1;
            sum += cnt[j];
        }
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    uint32_t run = incl - sum;
    constexpr uint32_t U = 32u * CH;
#pragma unroll
    for (int j = 0; j < kPer; j++) {
        const uint32_t i = i0 + j;
        if (i < n) {
            dd.sp_pre[i] = run;
            dd.sp_rec[i].x = q0s[j] - run;
            // the units that start inside this interval's chunks [run, run + cnt)
            const uint32_t ue = min((run + cnt[j] + U - 1u) / U, (uint32_t)kUnitTab);
            for (uint32_t u = (run + U - 1u) / U; u < ue; u++) sm.unit_k[u] = (uint8_t)i;
        }
        run += cnt[j];
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (lane == 0) {
        dd.sp_pre[n] = total;
        sm.next_unit = 0;
        sm.unit_n = min((total + U - 1u) / U, (uint32_t)kUnitTab);
    }
}

// Stream the ids of every interval of the span table into the scorecard.  Warps take
// units of 32 x CH consecutive 16-byte chunks (8 ids each) from a shared counter;
// lane l loads chunks l, l+32, ... of the unit, all before it scatters any.  The ids of
// a chunk outside its interval (at most the first and last chunk of an interval have
// some) are replaced through the keep masks: with the lane's dummy word when the tile
// is a whole block (every id of the block is then a word of the tile and needs no
// range check), else with 0xFFFF, which the range check sends to the dummy word
// (0xFFFF - lo >= lim: lo + lim <= 2 * block entries < 0xFFFF).
template <int CH>
__device__ __forceinline__ void stream_tile(BatchSmem &sm, const BatchDyn &dd, const uint4 *__restrict__ ia4,
                                            uint32_t ncv, void *scv, int ctile, bool wide, bool whole, uint32_t lo,
                                            uint32_t lim, int lane)
{
    const uint32_t M = dd.sp_pre[ncv];
    uint32_t *cnt = reinterpret_cast<uint32_t *>(scv);
    const uint32_t dummy = 2u * (uint32_t)ctile + (uint32_t)lane;   // packed: words [2T, 2T + 32)
    const uint32_t fill = whole ? (dummy | (dummy << 16)) : 0xFFFFFFFFu;
#if GX_STREAM_PREFETCH
    // The next unit's chunks are located and loaded before the current unit's ids are
    // scattered, so that the loads' latency overlaps the scatter.
    auto claim = [&]() -> uint32_t {
        uint32_t u = 0;
        if (lane == 0) u = atomicAdd(&sm.next_unit, 1u);
        return __shfl_sync(0xffffffffu, u, 0) * (32u * CH);
    };
    auto locate_load = [&](uint32_t j0, uint32_t (&kx)[CH], uint4 (&v)[CH]) {
        const uint32_t s1 = (uint32_t)lane * 8u;
        const uint32_t b1 = __ballot_sync(0xffffffffu, s1 < ncv && dd.sp_pre[s1] <= j0);
        const uint32_t base = (31u - (uint32_t)__clz(b1)) * 8u;
        const uint32_t s2 = base + ((uint32_t)lane & 7u);
        const uint32_t b2 = __ballot_sync(0xffffffffu, lane < 8 && s2 < ncv && dd.sp_pre[s2] <= j0);
        uint32_t k = base + (31u - (uint32_t)__clz(b2));
#pragma unroll
        for (int p = 0; p < CH; p++) {
            const uint32_t j = j0 + (uint32_t)lane + 32u * p;
            kx[p] = 0xFFFFFFFFu;
            if (j < M) {
                while (dd.sp_pre[k + 1] <= j) k++;
                kx[p] = k;
                v[p] = __ldg(ia4 + (dd.sp_rec[k].x + j));
            }
        }
    };
    uint32_t j0 = claim();
    uint4 v[CH];
    uint32_t kx[CH];
    if (j0 < M) locate_load(j0, kx, v);
    while (j0 < M) {
        const uint32_t jn = claim();
        uint4 vn[CH];
        uint32_t kn[CH];
        if (jn < M) locate_load(jn, kn, vn);
#pragma unroll
        for (int p = 0; p < CH; p++) {
            if (kx[p] == 0xFFFFFFFFu) continue;
            const uint4 r = dd.sp_rec[kx[p]];
            const uint32_t j = j0 + (uint32_t)lane + 32u * p;
            const uint32_t eq = (r.x + j) << 3;
            if (!wide) {
                const uint32_t mlo = r.y > eq ? r.y - eq : 0u;
                const uint32_t mhi = min(r.z - eq, 8u);
                const uint4 kl = sm.keep_lo[mlo], kh = sm.keep_hi[mhi - 1u];
                uint32_t w4[4] = {v[p].x, v[p].y, v[p].z, v[p].w};
                const uint32_t km[4] = {kl.x & kh.x, kl.y & kh.y, kl.z & kh.z, kl.w & kh.w};
#pragma unroll
                for (int q = 0; q < 4; q++) w4[q] = (w4[q] & km[q]) | (fill & ~km[q]);
                if (whole) {
#pragma unroll
                    for (int m = 0; m < 8; m++) atomicAdd(cnt + ((w4[m >> 1] >> (16 * (m & 1))) & 0xFFFFu), r.w);
                } else {
#pragma unroll
                    for (int m = 0; m < 8; m++)
                        scatter_packed(cnt, (w4[m >> 1] >> (16 * (m & 1))) & 0xFFFFu, lo, lim, r.w, dummy, true);
                }
            } else {
                const uint32_t c = dd.sp_c[kx[p]];
                const uint32_t w4[4] = {v[p].x, v[p].y, v[p].z, v[p].w};
                const bool full = eq >= r.y && eq + 8u <= r.z;
#pragma unroll
                for (int m = 0; m < 8; m++) {
                    const uint32_t e = eq + (uint32_t)m;
                    if (full || (e >= r.y && e < r.z))
                        scatter_wide(cnt, cnt + ctile, cnt + 2 * ctile, (w4[m >> 1] >> (16 * (m & 1))) & 0xFFFFu, lo,
                                     lim, c, r.w);
                }
            }
        }
        j0 = jn;
#pragma unroll
        for (int p = 0; p < CH; p++) {
            v[p] = vn[p];
            kx[p] = kn[p];
        }
    }
    return;
#endif
    for (;;) {
        uint32_t u = 0;
        if (lane == 0) u = atomicAdd(&sm.next_unit, 1u);
        u = __shfl_sync(0xffffffffu, u, 0);
        const uint32_t j0 = u * (32u * CH);
        if (j0 >= M) break;
        // interval of the unit's first chunk (the last k < ncv with pre[k] <= j0, a non-empty
        // interval: pre is non-decreasing, pre[0] = 0 and pre[ncv] > j0), recorded by the span
        // table's builder for the first units; each lane walks on from there
        uint32_t k;
        if (u < sm.unit_n) {
            k = sm.unit_k[u];
        } else {
#if GX_WARP_SEARCH
        // two levels across the warp: every 8th entry, then the 8 entries of that group
        const uint32_t s1 = (uint32_t)lane * 8u;
        const uint32_t b1 = __ballot_sync(0xffffffffu, s1 < ncv && dd.sp_pre[s1] <= j0);
        const uint32_t base = (31u - (uint32_t)__clz(b1)) * 8u;
        const uint32_t s2 = base + ((uint32_t)lane & 7u);
        const uint32_t b2 = __ballot_sync(0xffffffffu, lane < 8 && s2 < ncv && dd.sp_pre[s2] <= j0);
        k = base + (31u - (uint32_t)__clz(b2));
#else
        k = 0;
        uint32_t hi = ncv;
        while (hi - k > 1) {
            const uint32_t mid = (k + hi) >> 1;
            if (dd.sp_pre[mid] <= j0) k = mid; else hi = mid;
        }
#endif
        }
        uint4 v[CH];
        uint32_t kx[CH];
#pragma unroll
        for (int p = 0; p < CH; p++) {
            const uint32_t j = j0 + (uint32_t)lane + 32u * p;
            kx[p] = 0xFFFFFFFFu;
            if (j < M) {
                while (dd.sp_pre[k + 1] <= j) k++;
                kx[p] = k;
                v[p] = __ldg(ia4 + (dd.sp_rec[k].x + j));
            }
        }
#pragma unroll
        for (int p = 0; p < CH; p++) {
            if (kx[p] == 0xFFFFFFFFu) continue;
            const uint4 r = dd.sp_rec[kx[p]];
            const uint32_t j = j0 + (uint32_t)lane + 32u * p;
            const uint32_t eq = (r.x + j) << 3;   // element index of the chunk's first id
            if (!wide) {
                const uint32_t mlo = r.y > eq ? r.y - eq : 0u;      // 0..7
                const uint32_t mhi = min(r.z - eq, 8u);             // 1..8
                const uint4 kl = sm.keep_lo[mlo], kh = sm.keep_hi[mhi - 1u];
                uint32_t w4[4] = {v[p].x, v[p].y, v[p].z, v[p].w};
                const uint32_t km[4] = {kl.x & kh.x, kl.y & kh.y, kl.z & kh.z, kl.w & kh.w};
#pragma unroll
                for (int q = 0; q < 4; q++) w4[q] = (w4[q] & km[q]) | (fill & ~km[q]);
                if (whole) {
#pragma unroll
                    for (int m = 0; m < 8; m++) atomicAdd(cnt + ((w4[m >> 1] >> (16 * (m & 1))) & 0xFFFFu), r.w);
                } else {
#pragma unroll
                    for (int m = 0; m < 8; m++)
                        scatter_packed(cnt, (w4[m >> 1] >> (16 * (m & 1))) & 0xFFFFu, lo, lim, r.w, dummy, true);
                }
            } else {
                const uint32_t c = dd.sp_c[kx[p]];
                const uint32_t w4[4] = {v[p].x, v[p].y, v[p].z, v[p].w};
                const bool full = eq >= r.y && eq + 8u <= r.z;
#pragma unroll
                for (int m = 0; m < 8; m++) {
                    const uint32_t e = eq + (uint32_t)m;
                    if (full || (e >= r.y && e < r.z))
                        scatter_wide(cnt, cnt + ctile, cnt + 2 * ctile, (w4[m >> 1] >> (16 * (m & 1))) & 0xFFFFu, lo,
                                     lim, c, r.w);
                }
            }
        }
    }
}

// Whether k_search_piped takes spectrum s (k_search_batched takes the others).
__device__ __forceinline__ bool piped_spectrum(const SearchArgs &a, uint32_t s)
{
    const uint32_t nv = a.nivl[s];
    return a.guard[s] == 1u && nv >= 1u && nv <= (uint32_t)kIvlChunk && !(a.flags & GX_FLAG_WIDE_SCORECARD);
}

template <int CH>
__global__ void __launch_bounds__(kBBlock, kCtasPerSm) k_search_batched(SearchArgs a)
{
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ BatchSmem sm;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int i = tid; i < 81; i += kBBlock) sm.lgf[i] = a.lgfact[i];
    if (tid < 16) {   // keep masks (table lo: ids >= m; table hi: ids < m + 1)
        const int m = tid & 7;
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const bool k0 = tid < 8 ? 2 * q >= m : 2 * q < m + 1;
            const bool k1 = tid < 8 ? 2 * q + 1 >= m : 2 * q + 1 < m + 1;
            w[q] = (k0 ? 0x0000FFFFu : 0u) | (k1 ? 0xFFFF0000u : 0u);
        }
        (tid < 8 ? sm.keep_lo : sm.keep_hi)[m] = make_uint4(w[0], w[1], w[2], w[3]);
    }
    const int T = a.tile;
    void *scv = dyn;   // packed: T interleaved (b, y) word pairs; wide: 3 arrays of ctile words
    const BatchDyn dd = carve_dyn(dyn + (size_t)T * 8);
    for (int i = tid; i < 2 * T; i += kBBlock) reinterpret_cast<uint32_t *>(dyn)[i] = 0;
    // this warp's entrant list (global scratch, one slot per candidate of its range)
    Cell *ent = a.spill + ((uint64_t)blockIdx.x * kBWarps + wid) * (uint64_t)a.spill_per_warp;
    const uint32_t minshp = a.min_shp;

    for (;;) {
        __syncthreads();
        if (tid == 0) {
            int32_t spec = -1;
            for (;;) {   // with a.split, the spectra k_search_piped takes are left to it
                const uint32_t slot = atomicAdd(a.queue, 1u);
                if (slot >= a.nspec) break;
                const uint32_t s2 = a.order[slot];
                if (!a.split || !piped_spectrum(a, s2)) {
                    spec = (int32_t)s2;
                    break;
                }
            }
            sm.spec = spec;
            sm.heap_size = 0;
            sm.cpsms = 0;
            sm.status = 0;
            sm.root = 0.0f;
            sm.ent_mask = 0u;
            sm.ready = 0u;
        }
        for (int i = tid; i < kHist; i += kBBlock) sm.hist[i] = 0;
        __syncthreads();
        const int s = sm.spec;
        if (s < 0) break;
        if (a.nivl[s] == 0) {                 // no probed bins, or rejected by k_prep
            write_empty_row(a, a.hist_g, (uint32_t)s, a.guard[s] == kGuardRejected ? GX_STATUS_PEAK_LIMIT : 0, tid,
                            kBBlock);
            continue;
        }
        const bool wide = a.guard[s] == 0 || (a.flags & GX_FLAG_WIDE_SCORECARD);
        if (tid == 0 && wide) sm.status |= 8;
        const int ctile = wide ? ((T * 2) / 3) & ~31 : T;
        const uint32_t nv = a.nivl[s];
        const Interval *ivl = a.ivl + 2ull * a.qidx[s];
        int cps = 0;   // candidate PSMs counted by this warp (lane 0 adds them at the end)
        bool heap_due = false;
        // Offsets of the next tile's bins, loaded by thread i for interval i one tile ahead
        // (when all intervals fit one span table): the last warp builds that tile's span table from
        // them while the others score.
        uint32_t nx_s = 0, nx_e = 0;
        int nx_len = -1;
        int nx_kb = -1;
        const bool carry = nv <= (uint32_t)kIvlChunk;

        for (int ixx = 0; ixx < a.nlen; ixx++) {
            const int2 w = a.win[(uint64_t)s * a.nlen + ixx];
            if (w.y < w.x) continue;
            const DevLen ln = a.lens[ixx];
            const uint64_t base = ln.ia_off & ~7ull;              // 16-byte aligned
            const uint32_t rel0 = (uint32_t)(ln.ia_off - base);
            const uint4 *__restrict__ ia4 = reinterpret_cast<const uint4 *>(a.iAb + base);
            const uint32_t speclen = ln.speclen;
            constexpr int E = kBlockEntries;   // the index's block (launch_batched checks a.block)
            const int kb0 = w.x / E, kb1 = w.y / E;
            for (int kb = kb0; kb <= kb1; kb++) {
              // one block of entries = one candidate tile (two sub-tiles for the wide scorecard)
              const uint32_t *__restrict__ bA = a.blkA + ln.blk_off + (uint64_t)kb * (a.nbins + 1);
              const int bt0 = max(w.x, kb * E), bt1 = min(w.y + 1, (kb + 1) * E);
              const int nsub = (bt1 - bt0 + ctile - 1) / ctile;
              const bool have = carry && nx_len == ixx && nx_kb == kb;   // offsets loaded a tile ago
              const uint32_t cur_s = nx_s, cur_e = nx_e;
              // the next tile of this spectrum: the next block of this length, or the first
              // block of the next length with a window
              int nx = -1, nkb = 0;
              if (kb < kb1) {
                  nx = ixx;
                  nkb = kb + 1;
              } else {
                  for (int j = ixx + 1; j < a.nlen; j++) {
                      const int2 w2 = a.win[(uint64_t)s * a.nlen + j];
                      if (w2.y >= w2.x) {
                          nx = j;
                          nkb = w2.x / E;
                          break;
                      }
                  }
              }
              // (the next length's offsets are loaded only by the threads that use them: the
              // interval threads now, the last warp for the next span table after the scan)
              const bool has_next = carry && nx >= 0;
              if (has_next && tid < (int)nv) {
                  const uint64_t nblk = nx == ixx ? ln.blk_off : a.lens[nx].blk_off;
                  const uint32_t *nbA = a.blkA + nblk + (uint64_t)nkb * (a.nbins + 1);
                  const Interval v = ivl[tid];
                  nx_s = __ldg(nbA + v.b0);      // in flight while this tile streams
                  nx_e = __ldg(nbA + v.b1 + 1);
              }
              nx_len = nx;
              nx_kb = nkb;
              for (int ti = 0; ti < nsub; ti++) {
                const int t0 = bt0 + ti * ctile;
                const int t1 = min(bt1, t0 + ctile);
                const int tn = t1 - t0;
                if (tn <= 0) continue;
                const uint32_t lo = 2u * (uint32_t)(t0 - kb * E), lim = 2u * (uint32_t)tn;
                // the tile is the whole block (all its entries): every id of the block is a word of it
                const bool whole = !wide && t0 == kb * E && t1 == min((kb + 1) * E, (int)ln.npep);
                // ---- stream every interval's ids into the scorecard ----------------------
                const bool prebuilt = sm.ready != 0u;   // built while the last tile was scored
                for (uint32_t ic0 = 0; ic0 < nv; ic0 += kIvlChunk) {
                    const uint32_t ncv = min((uint32_t)kIvlChunk, nv - ic0);
                    if (!prebuilt) {
                        if (ti == 0 || nv > (uint32_t)kIvlChunk)
                            build_span_table(sm, dd, ivl + ic0, ncv, bA, rel0, have, cur_s, cur_e, wide, tid, lane,
                                             wid);
                        else if (tid == 0)
                            sm.next_unit = 0;
                        __syncthreads();
                    }
                    if (heap_due) {          // the previous tile's entrants, off the critical path
                        if (wid == kHeapWarp)
                            insert_entrants(sm, a.spill + (uint64_t)blockIdx.x * kBWarps * a.spill_per_warp,
                                            a.spill_per_warp, a.heap_cap, lane);
                        heap_due = false;
                    }
                    stream_tile<CH>(sm, dd, ia4, ncv, scv, ctile, wide, whole, lo, lim, lane);
                    if (ti == 0 && has_next && tid < (int)nv) {   // the next tile's offsets, for its span table
                        dd.nx_s[tid] = nx_s;
                        dd.nx_e[tid] = nx_e;
                    }
                    __syncthreads();
                }
                // ---- scan: warp w < kScanWarps owns candidates [w*R, (w+1)*R) and takes them ----
                // in entry order, four per lane per step, queues those that reach min_shp and
                // scores the queue when it is full and at the end; then clears its range for
                // the next tile.  Warp kHeapWarp builds the next tile's span table meanwhile.
                const float tau = sm.heap_size < a.heap_cap ? -1.0f : sm.root;
                const int step = wide ? 32 : 128;
                const int R = scan_range(tn, step);
                const int r0 = wid < kScanWarps ? min(tn, wid * R) : tn, r1 = min(tn, r0 + R);
                int npend = 0, nent = 0;
                uint32_t *sw = reinterpret_cast<uint32_t *>(scv);
                for (int c0 = r0; c0 < r1; c0 += step) {
                    unsigned m = 0;
                    int cb;
                    if (!wide) {
                        // lane l: candidates cb .. cb + 3 (cb = c0 + 4l), words b, y, b, y, b, y, b, y
                        cb = c0 + 4 * lane;
                        if (cb < r1) {
                            const uint4 qa = *reinterpret_cast<const uint4 *>(sw + 2 * cb);
                            const uint4 qb = *reinterpret_cast<const uint4 *>(sw + 2 * cb + 4);
                            const int lim4 = r1 - cb;   // candidates of the four inside the range
                            m = ((((qa.x >> 24) + (qa.y >> 24)) >= minshp) ? 1u : 0u) |
                                ((((qa.z >> 24) + (qa.w >> 24)) >= minshp) ? 2u : 0u) |
                                ((((qb.x >> 24) + (qb.y >> 24)) >= minshp) ? 4u : 0u) |
                                ((((qb.z >> 24) + (qb.w >> 24)) >= minshp) ? 8u : 0u);
                            if (lim4 < 4) m &= (1u << lim4) - 1u;
#if GX_FUSED_CLEAR
                            if (m == 0u) {   // no PSM among the four: reset them for the next tile now
                                uint4 *z = reinterpret_cast<uint4 *>(sw + 2 * cb);
                                z[0] = make_uint4(0u, 0u, 0u, 0u);
                                z[1] = make_uint4(0u, 0u, 0u, 0u);
                            }
#endif
                        }
                    } else {
                        cb = c0 + lane;
                        if (cb < r1) {
                            const uint32_t cv = sw[cb];
                            m = (((cv & 0xFFFFu) + (cv >> 16)) & 0xFFFFu) >= minshp ? 1u : 0u;
                        }
                    }
                    // queue positions: lane order, then candidate order inside the lane; the
                    // lanes' counts (0..4) by their three bits, one ballot each
                    const unsigned lt = (1u << lane) - 1u;
                    const unsigned nm = (unsigned)__popc(m);
                    const unsigned B0 = __ballot_sync(0xffffffffu, nm & 1u), B1 = __ballot_sync(0xffffffffu, nm & 2u);
                    const unsigned B2 = __ballot_sync(0xffffffffu, nm & 4u);
                    const int total = __popc(B0) + 2 * __popc(B1) + 4 * __popc(B2);
                    if (total == 0) continue;
                    if (npend + total > kPend) {   // queue full: score what it holds first
                        __syncwarp();
                        score_batch<BatchSmem, kEntSmem>(sm, dd.pend[wid], a, scv, ctile, wid, lane, npend, t0, ixx, speclen, tau, wide, ent,
                                                      nent, cps);
                        __syncwarp();
                        if (!wide && GX_FUSED_CLEAR) clear_scored(sw, dd.pend[wid], npend, lane);
                        npend = 0;
                        __syncwarp();
                    }
                    int pos = npend + __popc(B0 & lt) + 2 * __popc(B1 & lt) + 4 * __popc(B2 & lt);
                    for (unsigned mm = m; mm; mm &= mm - 1u) dd.pend[wid][pos++] = (uint32_t)(cb + __ffs(mm) - 1);
                    npend += total;
                }
                __syncwarp();
                if (npend > 0) {
                    score_batch<BatchSmem, kEntSmem>(sm, dd.pend[wid], a, scv, ctile, wid, lane, npend, t0, ixx, speclen, tau, wide, ent,
                                                      nent, cps);
                    __syncwarp();
                    if (!wide && GX_FUSED_CLEAR) clear_scored(sw, dd.pend[wid], npend, lane);
                }
                if (lane == 0) {
                    sm.warp_cnt[wid] = nent;
                    if (nent) atomicOr(&sm.ent_mask, 1u << wid);
                }
                // clear the warp's range [r0, r1) of every array (rounded up to 4 words: the
                // next range starts at a multiple of 32, the arrays end at one); the packed
                // scorecard was reset during the scan and after scoring
                __syncwarp();
                if (r0 < r1) {
                    if (!wide) {   // words [2 r0, 2 r1), two candidates per 16 bytes
                        if (!GX_FUSED_CLEAR) {
                            uint4 *z = reinterpret_cast<uint4 *>(sw);
                            for (int i = r0 / 2 + lane; i < (r1 + 1) / 2; i += 32) z[i] = make_uint4(0u, 0u, 0u, 0u);
                        }
                    } else {
                        const int q0 = r0 >> 2, q1 = min(ctile, (r1 + 3) & ~3) >> 2;
                        for (int k = 0; k < 3; k++) {
                            uint4 *z = reinterpret_cast<uint4 *>(sw + k * ctile);
                            for (int i = q0 + lane; i < q1; i += 32) z[i] = make_uint4(0u, 0u, 0u, 0u);
                        }
                    }
                }
                // the last warp prepares the next tile's span table (the others are still scoring)
                if (wid == kHeapWarp) {
                    if (ti + 1 < nsub && carry) {   // next sub-tile of this block: the same table, when one
                        if (lane == 0) { sm.next_unit = 0; sm.ready = 1u; }   // table holds every interval
                    } else if (ti + 1 >= nsub && has_next) {
                        const uint64_t nia = nx == ixx ? ln.ia_off : a.lens[nx].ia_off;
                        build_span_warp<CH>(sm, dd, nv, (uint32_t)(nia & 7ull), lane);
                        if (lane == 0) sm.ready = 1u;
                    } else if (lane == 0) {
                        sm.ready = 0u;
                    }
                }
                __syncthreads();
                heap_due = true;   // inserted by thread 0 while the next tile streams
              }
            }
        }
        if (heap_due && wid == kHeapWarp)
            insert_entrants(sm, a.spill + (uint64_t)blockIdx.x * kBWarps * a.spill_per_warp, a.spill_per_warp, a.heap_cap,
                            lane);
        if (lane == 0 && cps) atomicAdd(&sm.cpsms, cps);
        __syncthreads();
        // ---- per-spectrum outputs (the tail fit runs in k_tailfit) -------------------
        for (int i = tid; i < kHist; i += kBBlock) a.hist_g[(uint64_t)s * kHist + i] = sm.hist[i];
        if (a.heap_out)
            for (int i = tid; i < a.heap_cap; i += kBBlock) {
                gx_cell o{};
                if (i < sm.heap_size) {
                    const Cell c = sm.heap[i];
                    o.hyperscore = c.h; o.psid = c.psid; o.idxoffset = c.ixx; o.sharedions = c.shp;
                    o.totalions = c.total;
                }
                a.heap_out[(uint64_t)s * a.heap_cap + i] = o;
            }
        if (tid == 0) {
            gx_result r;
            memset(&r, 0, sizeof(r));
            r.cpsms = sm.cpsms;
            r.status = sm.status;
            if (fits_tail(sm.cpsms, a.min_cpsm)) {
                const Cell t = heap_getmax(sm.heap, sm.heap_size);
                r.top.hyperscore = t.h; r.top.psid = t.psid; r.top.idxoffset = t.ixx;
                r.top.sharedions = t.shp; r.top.totalions = t.total;
                r.maxhyp = __double2int_rz(__dadd_rn((double)__fmul_rn(t.h, 10.0f), 0.5));
            }
            a.out[s] = r;
        }
    }
}


// ------------------------------------------------------------------------------------
// k_search_piped: one CTA of 32 warps per SM with two scorecard tiles.  In phase p every
// warp scans and scores its range of tile p - 1 (one buffer), then takes work units of
// tile p's ids (the other buffer) until none are left; warp 0 prepares tile p + 1 (its
// descriptor and span table) and the last warp first inserts tile p - 2's heap entrants.
// One barrier per tile, and the stream's dynamic units absorb the uneven scoring.  It
// takes the spectra with the 8-byte scorecard and at most kIvlChunk intervals (almost all
// of them); k_search_batched takes the rest in a second launch.
// ------------------------------------------------------------------------------------
constexpr int kPWarps = 32;
// Candidates of a tile of tn that each warp of k_search_piped scans (a multiple of 128): at
// most the length of the warp's entrant list of one tile parity.
__host__ __device__ constexpr int piped_range(int tn) { return ((tn + kPWarps - 1) / kPWarps + 127) / 128 * 128; }
constexpr int kPBlock = kPWarps * 32;
constexpr int kPPend = 136;                  // per-warp queue: one scan step (128) + slack
constexpr int kPHeapWarp = kPWarps - 1;
static_assert(kPPend >= 128, "the queue must hold one scan step's candidates (32 lanes x 4)");

struct PipedTile {
    int32_t valid;
    int32_t ixx;
    int32_t t0, tn;
    uint32_t lo, lim;       // block-local id range of the tile: id - lo < lim
    int32_t whole;          // the tile is its whole block
    uint32_t speclen;
    uint64_t base;          // 16-byte aligned element offset of the length's ids in iAb
};

struct PipedSmem {
    uint32_t hist[kHist];
    double lgf[81];
    Cell heap[kMaxHeap + 1];
    int32_t warp_cnt[2][kPWarps];   // entrants per warp, by tile parity
    uint32_t ent_mask[2];
    uint32_t next_unit[2];          // work-unit counter of the tile streaming into buffer b
    int32_t heap_size;
    int32_t cpsms;
    int32_t status;
    int32_t spec;
    float tau;                      // entrant threshold: -1 while the heap is not full, then its root
    int32_t it_ixx;                 // tile iterator (written by warp 0)
    int64_t it_kb, it_kb1;
    uint4 keep_lo[8];
    uint4 keep_hi[8];
    PipedTile tile[3];              // tiles p - 1 (scanned), p (streamed), p + 1 (prepared): by tile number mod 3
};

struct PipedDyn {
    uint32_t *card[2];              // scorecard words [2T] + kDummy dummy words, per buffer
    uint32_t (*pend)[kPPend];
    uint4 *sp_rec[2];
    uint32_t *sp_pre[2];
};

__host__ __device__ constexpr size_t piped_card_words(int tile) { return 2 * (size_t)tile + kDummy; }

__host__ __device__ constexpr size_t piped_dyn_bytes(int tile)
{
    return sizeof(uint32_t) * (2 * piped_card_words(tile) + (size_t)kPWarps * kPPend +
                               2 * (4 * (size_t)kIvlChunk + (kIvlChunk + 4)));
}

__device__ __forceinline__ PipedDyn carve_piped(unsigned char *base, int tile)
{
    PipedDyn d;
    uint32_t *p = reinterpret_cast<uint32_t *>(base);
    d.card[0] = p; p += piped_card_words(tile);
    d.card[1] = p; p += piped_card_words(tile);
    d.pend = reinterpret_cast<uint32_t (*)[kPPend]>(p); p += (size_t)kPWarps * kPPend;
    for (int b = 0; b < 2; b++) {   // 16-byte aligned: every block above is a multiple of 4 words
        d.sp_rec[b] = reinterpret_cast<uint4 *>(p); p += 4 * kIvlChunk;
        d.sp_pre[b] = p; p += kIvlChunk + 4;
    }
    return d;
}

// Warp 0: the next tile of spectrum s (the next entry block of the current length's window,
// or the first block of the next length with a window) into slot `slot`, with its span table
// in buffer b: per interval, its chunk offset, id range and add value, and the exclusive
// prefix of the intervals' 16-byte chunk counts.  Resets buffer b's unit counter.
__device__ void piped_prepare(PipedSmem &sm, const PipedDyn &dd, const SearchArgs &a, int s, const Interval *ivl,
                              uint32_t nv, int slot, int b, int lane)
{
    int ixx = sm.it_ixx;
    int64_t kb = sm.it_kb + 1, kb1 = sm.it_kb1;
    const int64_t E = a.block;
    if (kb > kb1) {
        for (ixx = ixx + 1; ixx < a.nlen; ixx++) {
            const int2 w = a.win[(uint64_t)s * a.nlen + ixx];
            if (w.y >= w.x) {
                kb = w.x / E;
                kb1 = w.y / E;
                break;
            }
        }
    }
    __syncwarp();
    if (ixx >= a.nlen) {
        if (lane == 0) {
            sm.tile[slot].valid = 0;
            sm.it_ixx = ixx;
        }
        return;
    }
    const int2 w = a.win[(uint64_t)s * a.nlen + ixx];
    const DevLen ln = a.lens[ixx];
    const int t0 = (int)max((int64_t)w.x, kb * E), t1 = (int)min((int64_t)w.y + 1, (kb + 1) * E);
    const uint64_t base = ln.ia_off & ~7ull;
    const uint32_t rel0 = (uint32_t)(ln.ia_off - base);
    const uint32_t *__restrict__ bA = a.blkA + ln.blk_off + (uint64_t)kb * (a.nbins + 1);
    constexpr int kPer = kIvlChunk / 32;
    uint32_t cnt[kPer], q0s[kPer];
    uint32_t sum = 0;
#pragma unroll
    for (int j = 0; j < kPer; j++) {
        const uint32_t i = (uint32_t)lane * kPer + j;
        cnt[j] = 0;
        q0s[j] = 0;
        if (i < nv) {
            const Interval v = ivl[i];
            const uint32_t a0 = rel0 + __ldg(bA + v.b0), a1 = rel0 + __ldg(bA + v.b1 + 1);
            const uint32_t q0 = a0 >> 3;
            cnt[j] = a1 > a0 ? ((a1 + 7u) >> 3) - q0 : 0u;
            q0s[j] = q0;
            dd.sp_rec[b][i] = make_uint4(0u, a0, a1, (v.c << 24) | v.S);
            sum += cnt[j];
        }
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    uint32_t run = incl - sum;
#pragma unroll
    for (int j = 0; j < kPer; j++) {
        const uint32_t i = (uint32_t)lane * kPer + j;
        if (i < nv) {
            dd.sp_pre[b][i] = run;
            dd.sp_rec[b][i].x = q0s[j] - run;
        }
        run += cnt[j];
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (lane == 0) {
        dd.sp_pre[b][nv] = total;
        sm.next_unit[b] = 0;
        PipedTile t;
        t.valid = 1;
        t.ixx = ixx;
        t.t0 = t0;
        t.tn = t1 - t0;
        t.lo = 2u * (uint32_t)(t0 - kb * E);
        t.lim = 2u * (uint32_t)(t1 - t0);
        t.whole = ((int64_t)t0 == kb * E && (int64_t)t1 == min((kb + 1) * E, (int64_t)ln.npep)) ? 1 : 0;
        t.speclen = ln.speclen;
        t.base = base;
        sm.tile[slot] = t;
        sm.it_ixx = ixx;
        sm.it_kb = kb;
        sm.it_kb1 = kb1;
    }
}

// The ids of every interval of a span table into an 8-byte scorecard (stream_tile's packed
// path: units of 32 x CH 16-byte chunks from a shared counter, keep masks for the ids of
// an interval's first and last chunk that lie outside it, the lane's dummy word for ids
// outside the tile).
template <int CH>
__device__ __forceinline__ void piped_stream(uint32_t *next_unit, const uint4 *keep_lo, const uint4 *keep_hi,
                                             const uint4 *sp_rec, const uint32_t *sp_pre,
                                             const uint4 *__restrict__ ia4, uint32_t ncv, uint32_t *cnt, int ctile,
                                             bool whole, uint32_t lo, uint32_t lim, int lane)
{
    const uint32_t M = sp_pre[ncv];
    const uint32_t dummy = 2u * (uint32_t)ctile + (uint32_t)lane;
    const uint32_t fill = whole ? (dummy | (dummy << 16)) : 0xFFFFFFFFu;
    for (;;) {
        uint32_t u = 0;
        if (lane == 0) u = atomicAdd(next_unit, 1u);
        u = __shfl_sync(0xffffffffu, u, 0);
        const uint32_t j0 = u * (32u * CH);
        if (j0 >= M) break;
        const uint32_t s1 = (uint32_t)lane * 8u;
        const uint32_t b1 = __ballot_sync(0xffffffffu, s1 < ncv && sp_pre[s1] <= j0);
        const uint32_t base = (31u - (uint32_t)__clz(b1)) * 8u;
        const uint32_t s2 = base + ((uint32_t)lane & 7u);
        const uint32_t b2 = __ballot_sync(0xffffffffu, lane < 8 && s2 < ncv && sp_pre[s2] <= j0);
        uint32_t k = base + (31u - (uint32_t)__clz(b2));
        uint4 v[CH];
        uint32_t kx[CH];
#pragma unroll
        for (int p = 0; p < CH; p++) {
            const uint32_t j = j0 + (uint32_t)lane + 32u * p;
            kx[p] = 0xFFFFFFFFu;
            if (j < M) {
                while (sp_pre[k + 1] <= j) k++;
                kx[p] = k;
                v[p] = __ldg(ia4 + (sp_rec[k].x + j));
            }
        }
#pragma unroll
        for (int p = 0; p < CH; p++) {
            if (kx[p] == 0xFFFFFFFFu) continue;
            const uint4 r = sp_rec[kx[p]];
            const uint32_t j = j0 + (uint32_t)lane + 32u * p;
            const uint32_t eq = (r.x + j) << 3;
            const uint32_t mlo = r.y > eq ? r.y - eq : 0u;
            const uint32_t mhi = min(r.z - eq, 8u);
            const uint4 kl = keep_lo[mlo], kh = keep_hi[mhi - 1u];
            uint32_t w4[4] = {v[p].x, v[p].y, v[p].z, v[p].w};
            const uint32_t km[4] = {kl.x & kh.x, kl.y & kh.y, kl.z & kh.z, kl.w & kh.w};
#pragma unroll
            for (int q = 0; q < 4; q++) w4[q] = (w4[q] & km[q]) | (fill & ~km[q]);
            if (whole) {
#pragma unroll
                for (int m = 0; m < 8; m++) atomicAdd(cnt + ((w4[m >> 1] >> (16 * (m & 1))) & 0xFFFFu), r.w);
            } else {
#pragma unroll
                for (int m = 0; m < 8; m++)
                    scatter_packed(cnt, (w4[m >> 1] >> (16 * (m & 1))) & 0xFFFFu, lo, lim, r.w, dummy, true);
            }
        }
    }
}

// Warp kPHeapWarp: the entrants of the tile of parity `par` into the heap, in warp order
// (each warp's list is in candidate order), as insert_entrants does (lists in global memory).
__device__ __noinline__ void piped_insert(PipedSmem &sm, const Cell *lists, uint32_t stride, int par, int cap,
                                          int lane)
{
    int hs = sm.heap_size;
    for (uint32_t mask = sm.ent_mask[par]; mask; mask &= mask - 1u) {
        const int w2 = __ffs(mask) - 1;
        const int n2 = sm.warp_cnt[par][w2];
        const Cell *e2 = lists + ((uint64_t)par * kPWarps + w2) * stride;
        Cell nxt;
        if (lane < n2) nxt = e2[lane];
        for (int k0 = 0; k0 < n2; k0 += 32) {
            const Cell c = nxt;
            const bool v = k0 + lane < n2;
            const int k1 = k0 + 32 + lane;
            if (k1 < n2) nxt = e2[k1];
            __syncwarp();
            const float root = hs == cap ? sm.heap[0].h : -INFINITY;
            uint32_t live = __ballot_sync(0xffffffffu, v && c.h >= root);
            const uint32_t u1 = ((uint32_t)c.ixx) | ((uint32_t)c.shp << 16);
            const uint32_t u2 = ((uint32_t)c.total) | ((uint32_t)c.pad << 16);
            while (live) {
                const int j = __ffs(live) - 1;
                live &= live - 1u;
                Cell cj;
                cj.h = __shfl_sync(0xffffffffu, c.h, j);
                cj.psid = __shfl_sync(0xffffffffu, c.psid, j);
                const uint32_t v1 = __shfl_sync(0xffffffffu, u1, j), v2 = __shfl_sync(0xffffffffu, u2, j);
                cj.ixx = (uint16_t)(v1 & 0xFFFFu); cj.shp = (uint16_t)(v1 >> 16);
                cj.total = (uint16_t)(v2 & 0xFFFFu); cj.pad = (uint16_t)(v2 >> 16);
                if (lane == 0) {
                    int h0 = hs;
                    heap_insert(sm.heap, h0, cap, cj);
                }
                hs = min(hs + 1, cap);
            }
        }
    }
    __syncwarp();
    if (lane == 0) {
        sm.heap_size = hs;
        sm.ent_mask[par] = 0u;
        *reinterpret_cast<volatile float *>(&sm.tau) = hs == cap ? sm.heap[0].h : -1.0f;
    }
}

template <int CH>
__global__ void __launch_bounds__(kPBlock, 1) k_search_piped(SearchArgs a)
{
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ PipedSmem sm;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int i = tid; i < 81; i += kPBlock) sm.lgf[i] = a.lgfact[i];
    if (tid < 16) {   // keep masks (table lo: ids >= m; table hi: ids < m + 1)
        const int m = tid & 7;
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const bool k0 = tid < 8 ? 2 * q >= m : 2 * q < m + 1;
            const bool k1 = tid < 8 ? 2 * q + 1 >= m : 2 * q + 1 < m + 1;
            w[q] = (k0 ? 0x0000FFFFu : 0u) | (k1 ? 0xFFFF0000u : 0u);
        }
        (tid < 8 ? sm.keep_lo : sm.keep_hi)[m] = make_uint4(w[0], w[1], w[2], w[3]);
    }
    const int T = a.tile;   // the index's block: every tile is (part of) one block
    const PipedDyn dd = carve_piped(dyn, T);
    for (size_t i = tid; i < 2 * piped_card_words(T); i += kPBlock) dd.card[0][i] = 0u;
    // entrant lists of this CTA: [parity][warp][stride]
    const uint32_t stride = a.spill_per_warp / 2u;
    const Cell *lists = a.spill + (uint64_t)blockIdx.x * 2 * kPWarps * stride;
    const uint32_t minshp = a.min_shp;

    for (;;) {
        __syncthreads();
        if (tid == 0) {
            int spec = -1;
            for (;;) {
                const uint32_t slot = atomicAdd(a.queue, 1u);
                if (slot >= a.nspec) break;
                const uint32_t s = a.order[slot];
                if (piped_spectrum(a, s)) {
                    spec = (int)s;
                    break;
                }
            }
            sm.spec = spec;
            sm.heap_size = 0;
            sm.cpsms = 0;
            sm.status = 0;
            sm.tau = -1.0f;
            sm.ent_mask[0] = sm.ent_mask[1] = 0u;
            sm.it_ixx = -1;
            sm.it_kb = 0;
            sm.it_kb1 = -1;
        }
        for (int i = tid; i < kHist; i += kPBlock) sm.hist[i] = 0;
        __syncthreads();
        const int s = sm.spec;
        if (s < 0) break;
        const uint32_t nv = a.nivl[s];
        const Interval *ivl = a.ivl + 2ull * a.qidx[s];
        if (wid == 0) piped_prepare(sm, dd, a, s, ivl, nv, 0, 0, lane);
        __syncthreads();
        int cps = 0;
        int last_par = -1;   // parity of the last scanned tile (its entrants wait for the end)
        for (int p = 0;; p++) {
            const int bs = (p + 1) & 1, bt = p & 1;   // buffers of tiles p - 1 and p
            const PipedTile ts = sm.tile[(p + 2) % 3], tt = sm.tile[p % 3];
            const bool scan = p > 0 && ts.valid;
            const bool strm = tt.valid != 0;
            if (!scan && !strm) break;
            if (wid == kPHeapWarp && p >= 2) piped_insert(sm, lists, stride, bt, a.heap_cap, lane);
            if (scan) {
                // ---- scan and score tile p - 1: warp w owns [w R, (w + 1) R), four candidates per lane per step
                const float tau = *reinterpret_cast<volatile float *>(&sm.tau);
                const int tn = ts.tn;
                const int R = piped_range(tn);
                const int r0 = min(tn, wid * R), r1 = min(tn, r0 + R);
                uint32_t *sw = dd.card[bs];
                uint32_t *pend = dd.pend[wid];
                Cell *ent = const_cast<Cell *>(lists) + ((uint64_t)bs * kPWarps + wid) * stride;
                int npend = 0, nent = 0;
                for (int c0 = r0; c0 < r1; c0 += 128) {
                    unsigned m = 0;
                    const int cb = c0 + 4 * lane;
                    if (cb < r1) {
                        uint4 *z = reinterpret_cast<uint4 *>(sw + 2 * cb);
                        const uint4 qa = z[0], qb = z[1];
                        const int lim4 = r1 - cb;
                        m = ((((qa.x >> 24) + (qa.y >> 24)) >= minshp) ? 1u : 0u) |
                            ((((qa.z >> 24) + (qa.w >> 24)) >= minshp && lim4 > 1) ? 2u : 0u) |
                            ((((qb.x >> 24) + (qb.y >> 24)) >= minshp && lim4 > 2) ? 4u : 0u) |
                            ((((qb.z >> 24) + (qb.w >> 24)) >= minshp && lim4 > 3) ? 8u : 0u);
                        if (m == 0u) {   // no PSM among the four: reset them for the tile after next
                            z[0] = make_uint4(0u, 0u, 0u, 0u);
                            z[1] = make_uint4(0u, 0u, 0u, 0u);
                        }
                    }
                    const unsigned lt = (1u << lane) - 1u;
                    const unsigned B0 = __ballot_sync(0xffffffffu, m & 1u), B1 = __ballot_sync(0xffffffffu, m & 2u);
                    const unsigned B2 = __ballot_sync(0xffffffffu, m & 4u), B3 = __ballot_sync(0xffffffffu, m & 8u);
                    const int total = __popc(B0) + __popc(B1) + __popc(B2) + __popc(B3);
                    if (total == 0) continue;
                    if (npend + total > kPPend) {
                        __syncwarp();
                        score_batch<PipedSmem, 0>(sm, pend, a, sw, T, wid, lane, npend, ts.t0, ts.ixx, ts.speclen, tau,
                                                  false, ent, nent, cps);
                        __syncwarp();
                        for (int i = lane; i < npend; i += 32) {
                            uint4 *z = reinterpret_cast<uint4 *>(sw + 2 * (pend[i] & ~3u));
                            z[0] = make_uint4(0u, 0u, 0u, 0u);
                            z[1] = make_uint4(0u, 0u, 0u, 0u);
                        }
                        npend = 0;
                        __syncwarp();
                    }
                    int pos = npend + __popc(B0 & lt) + __popc(B1 & lt) + __popc(B2 & lt) + __popc(B3 & lt);
                    for (unsigned mm = m; mm; mm &= mm - 1u) pend[pos++] = (uint32_t)(cb + __ffs(mm) - 1);
                    npend += total;
                }
                __syncwarp();
                if (npend > 0) {
                    score_batch<PipedSmem, 0>(sm, pend, a, sw, T, wid, lane, npend, ts.t0, ts.ixx, ts.speclen, tau,
                                              false, ent, nent, cps);
                    __syncwarp();
                    for (int i = lane; i < npend; i += 32) {
                        uint4 *z = reinterpret_cast<uint4 *>(sw + 2 * (pend[i] & ~3u));
                        z[0] = make_uint4(0u, 0u, 0u, 0u);
                        z[1] = make_uint4(0u, 0u, 0u, 0u);
                    }
                }
                if (lane == 0) {
                    sm.warp_cnt[bs][wid] = nent;
                    if (nent) atomicOr(&sm.ent_mask[bs], 1u << wid);
                }
                last_par = bs;
            }
            // ---- warp 0 prepares tile p + 1 (slot (p + 1) mod 3, buffer bs: tile p - 1's)
            if (wid == 0) piped_prepare(sm, dd, a, s, ivl, nv, (p + 1) % 3, bs, lane);
            // ---- stream tile p into buffer bt
            if (strm) {
                const uint4 *__restrict__ ia4 = reinterpret_cast<const uint4 *>(a.iAb + tt.base);
                piped_stream<CH>(&sm.next_unit[bt], sm.keep_lo, sm.keep_hi, dd.sp_rec[bt], dd.sp_pre[bt], ia4, nv,
                                 dd.card[bt], T, tt.whole != 0, tt.lo, tt.lim, lane);
            }
            __syncthreads();
        }
        if (last_par >= 0 && wid == kPHeapWarp) piped_insert(sm, lists, stride, last_par, a.heap_cap, lane);
        if (lane == 0 && cps) atomicAdd(&sm.cpsms, cps);
        __syncthreads();
        // ---- per-spectrum outputs (the tail fit runs in k_tailfit)
        for (int i = tid; i < kHist; i += kPBlock) a.hist_g[(uint64_t)s * kHist + i] = sm.hist[i];
        if (a.heap_out)
            for (int i = tid; i < a.heap_cap; i += kPBlock) {
                gx_cell o{};
                if (i < sm.heap_size) {
                    const Cell c = sm.heap[i];
                    o.hyperscore = c.h; o.psid = c.psid; o.idxoffset = c.ixx; o.sharedions = c.shp;
                    o.totalions = c.total;
                }
                a.heap_out[(uint64_t)s * a.heap_cap + i] = o;
            }
        if (tid == 0) {
            gx_result r;
            memset(&r, 0, sizeof(r));
            r.cpsms = sm.cpsms;
            r.status = sm.status;
            if (fits_tail(sm.cpsms, a.min_cpsm)) {
                const Cell t = heap_getmax(sm.heap, sm.heap_size);
                r.top.hyperscore = t.h; r.top.psid = t.psid; r.top.idxoffset = t.ixx;
                r.top.sharedions = t.shp; r.top.totalions = t.total;
                r.maxhyp = __double2int_rz(__dadd_rn((double)__fmul_rn(t.h, 10.0f), 0.5));
            }
            a.out[s] = r;
        }
    }
}

// ------------------------------------------------------------------------------------
// k_tailfit: one warp per spectrum (the FP64 fit itself is serial in lane 0)
// ------------------------------------------------------------------------------------
constexpr int kTfWarps = 4;

__global__ void __launch_bounds__(kTfWarps * 32) k_tailfit(SearchArgs a)
{
    __shared__ uint32_t h[kTfWarps][kHist];
    __shared__ double sx[kTfWarps][kHist + 2];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t s = blockIdx.x * kTfWarps + w;
    if (s >= a.nspec) return;
    gx_result r = a.out[s];
    if (!fits_tail(r.cpsms, a.min_cpsm)) return;
    for (int i = lane; i < kHist; i += 32) h[w][i] = a.hist_g[(uint64_t)s * kHist + i];
    __syncwarp();
    tail_fit_warp(h[w], r.cpsms, r.maxhyp, sx[w], r, lane);
    if (lane == 0) {
        r.status |= 1;
        if (r.e_x < a.expect_max) r.status |= 2;
        a.out[s] = r;
    }
}

// ------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------
size_t batched_sort_temp_bytes(uint32_t max_spec)
{
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, (const uint64_t *)nullptr, (uint64_t *)nullptr,
                                              (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)max_spec);
    return bytes;
}

__global__ void k_logtab(double *tab, uint32_t n)
{
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n) tab[x] = log10((double)x);
}

cudaError_t fill_logtab(double *tab, uint32_t n, cudaStream_t st)
{
    k_logtab<<<(n + 255) / 256, 256, 0, st>>>(tab, n);
    count_launch();
    return cudaGetLastError();
}

size_t batched_dyn_smem(int tile) { return (size_t)tile * 8 + batch_dyn_bytes(tile); }

namespace {
using SearchKernel = void (*)(SearchArgs);
SearchKernel search_kernel(int chunks)
{
    switch (chunks) {
    case 1: return k_search_batched<1>;
    case 3: return k_search_batched<3>;
    default: return k_search_batched<2>;
    }
}
SearchKernel piped_kernel(int chunks)
{
    switch (chunks) {
    case 1: return k_search_piped<1>;
    case 3: return k_search_piped<3>;
    default: return k_search_piped<2>;
    }
}
}  // namespace

// Whether one CTA of k_search_piped<chunks> fits an SM at this tile size.
bool piped_fits(int tile, int chunks)
{
    int n = 0;
    if (cudaFuncSetAttribute(piped_kernel(chunks), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)piped_dyn_bytes(tile)) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, piped_kernel(chunks), kPBlock, piped_dyn_bytes(tile)) !=
        cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return n >= 1;
}

// CTAs of k_search_batched<chunks> that fit one SM at this tile size (at most kCtasPerSm).
int batched_ctas_per_sm(int tile, int chunks)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, search_kernel(chunks), kBBlock, batched_dyn_smem(tile)) !=
        cudaSuccess)
        n = 1;
    return n < 1 ? 1 : (n > kCtasPerSm ? kCtasPerSm : n);
}

// Largest candidate range of one warp in a tile (its entrants never exceed it).
uint32_t batched_spill_per_warp(int tile)
{
    // the largest range of k_search_batched: the 8-byte scorecard's (step 128) over the whole
    // tile (the 12-byte scorecard's ranges, step 32 over two thirds of it, are shorter); and
    // k_search_piped's, which keeps two lists (one per tile parity) in the same space
    const int r = scan_range(tile, 128), rp = 2 * piped_range(tile);
    return (uint32_t)(r > rp ? r : rp);
}

cudaError_t batched_set_attributes(int tile)
{
    cudaError_t e = cudaSuccess;
    for (int c = 1; c <= kMaxChunks && e == cudaSuccess; c++)
        e = cudaFuncSetAttribute(search_kernel(c), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)batched_dyn_smem(tile));
    return e;
}

bool batched_tiles_valid(const BatchedTiles &t, int max_tile)
{
    return t.chunks >= 1 && t.chunks <= kMaxChunks && t.ctas_per_sm >= 1 && t.ctas_per_sm <= kCtasPerSm &&
           t.tile >= kMinTile && t.tile <= max_tile && t.tile % 32 == 0 && (t.sorted == 0 || t.sorted == 1) &&
           (t.pipeline == 0 || (t.pipeline == 1 && t.tile == max_tile));
}

cudaError_t launch_batched(SearchArgs a, const BatchedScratch &b, const BatchedTiles &t, cudaStream_t st)
{
    cudaError_t e;
    if (a.block != (uint32_t)kBlockEntries) return cudaErrorInvalidValue;   // k_search_batched's tile arithmetic
    a.tile = t.tile;
    int h = prof_begin("k_prep", st);
    k_prep<<<a.nspec, kPrepBlock, 0, st>>>(a, const_cast<int2 *>(a.win), b.key_in, b.ord_in);
    prof_end(h, st);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    a.order = b.ord_in;   // batch order
    if (t.sorted) {       // heaviest scan volume first
        size_t tb = b.sort_temp_bytes;
        h = prof_begin("sort_by_volume", st);
        e = cub::DeviceRadixSort::SortPairsDescending(b.sort_temp, tb, b.key_in, b.key_out, b.ord_in, b.ord_out,
                                                      (int)a.nspec, 0, 64, st);
        prof_end(h, st);
        count_launch();
        if (e != cudaSuccess) return e;
        a.order = b.ord_out;
    }
    if ((e = cudaMemsetAsync(a.queue, 0, 2 * sizeof(uint32_t), st)) != cudaSuccess) return e;
    if (t.pipeline) {   // the pipelined kernel first, on its own queue counter; the batched one takes the rest
        SearchArgs ap = a;
        ap.queue = a.queue + 1;
        h = prof_begin("k_search_piped", st);
        piped_kernel(t.chunks)<<<b.sms, kPBlock, piped_dyn_bytes(a.tile), st>>>(ap);
        prof_end(h, st);
        count_launch();
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        a.split = 1;
    }
    const int ctas = t.ctas_per_sm < b.max_ctas[t.chunks] ? t.ctas_per_sm : b.max_ctas[t.chunks];
    h = prof_begin("k_search_batched", st);
    search_kernel(t.chunks)<<<b.sms * ctas, kBBlock, batched_dyn_smem(a.tile), st>>>(a);
    prof_end(h, st);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    h = prof_begin("k_tailfit", st);
    k_tailfit<<<(a.nspec + kTfWarps - 1) / kTfWarps, kTfWarps * 32, 0, st>>>(a);
    prof_end(h, st);
    count_launch();
    return cudaGetLastError();
}

}  // namespace gx
