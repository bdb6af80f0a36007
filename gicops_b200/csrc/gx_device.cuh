// Device-side building blocks of the query path shared by the search kernels.
#pragma once

#include <cstdint>
#include <cstring>

#include "../../include/gicops_b200.h"

namespace gx {

constexpr int kHist = GX_HIST_BINS;
constexpr int kMaxHeap = GX_MAX_HEAP;

// Per-length constants of a device-resident index.
struct DevLen {
    uint64_t ia_off;      // first ion id of this length in the concatenated iA
    uint64_t mass_off;    // first entry of this length in the concatenated masses
    uint32_t npep;        // entries
    uint32_t speclen;     // ions per entry
    uint32_t half;        // speclen / 2 (b ions first, then y ions)
    uint32_t peplen;
    uint32_t magic;       // ceil(2^32 / speclen): id / speclen = umulhi(id, magic), minus one if over
    uint32_t nblk;        // entry blocks of the block layout
    uint64_t blk_off;     // first offset table of this length in blkA
};

// Exact id / speclen for any 32-bit id: umulhi with ceil(2^32/d) is at most one too large.
__device__ __forceinline__ uint32_t div_speclen(uint32_t id, uint32_t d, uint32_t magic)
{
    uint32_t q = __umulhi(id, magic);
    if ((uint64_t)q * d > id) q--;
    return q;
}

// A run of consecutive fragment bins [b0, b1] covered by the same set of peak
// windows: c peaks, intensity sum S (mod 2^32).
struct Interval {
    uint32_t b0, b1;
    uint32_t c;
    uint32_t S;
};

// One heap cell as kept on chip.
struct Cell {
    float h;
    int32_t psid;
    uint16_t ixx;
    uint16_t shp;
    uint16_t total;
    uint16_t pad;
};

// Everything a search launch reads.
struct SearchArgs {
    // index
    const uint32_t *bA;   // [nlen * nbins]
    const uint32_t *iA;   // bin-major CSR ids (device form 2*entry + y)
    const uint16_t *iAb;  // block layout: per block of `block` entries, a CSR over bins of
                          // block-local ids 2*(entry - block start) + (y ion)
    const uint32_t *blkA; // block layout offsets [nblk][nbins + 1] per length (relative to ia_off)
    uint32_t block;       // entries per block
    uint64_t iab_bytes;   // bytes of ids in iAb (the allocation adds one 16-byte chunk)
    const float *mass;
    const DevLen *lens;
    int32_t nlen;
    uint32_t nbins;
    uint32_t maxz;
    // queries
    const uint32_t *qidx;
    const int32_t *moz;
    const int32_t *intn;
    const float *prec;
    const double *dMq;
    uint32_t nspec;
    // parameters
    double dM;
    double upper;         // peaks need (double)m/z < upper = max_mass*scale - 1 - dF
    uint32_t dF;
    uint32_t min_shp;
    uint32_t min_cpsm;
    int32_t heap_cap;
    double expect_max;
    uint32_t flags;
    const double *lgfact; // [81]
    const double *logtab; // [logtab_n]: log10(x) for small integers x
    uint32_t logtab_n;
    // scratch / outputs
    const int2 *win;      // [nspec * nlen] candidate window per (spectrum, length)
    // batched path
    Interval *ivl;        // [2 * npeaks]: intervals of spectrum s start at 2 * qidx[s]
    uint64_t ivl_cap;     // intervals the buffer holds
    uint32_t *nivl;       // [nspec]
    uint32_t *guard;      // [nspec]: 1 if the packed scorecard is exact for the spectrum, 0 if not,
                          // 2 if the spectrum was rejected (not searched)
    const uint32_t *order;// [nspec] spectra, heaviest first
    uint32_t *queue;      // work-queue head (two counters: the batched and the pipelined kernel)
    uint32_t split;       // 1: k_search_batched leaves the spectra k_search_piped takes
    uint32_t *hist_g;     // [nspec * kHist] histograms (always)
    int32_t tile;         // candidates per scorecard tile
    Cell *spill;          // [grid * 32 warps * spill_per_warp] heap entrants of each warp's range
    uint32_t spill_per_warp;
    gx_result *out;
    gx_cell *heap_out;    // optional [nspec * heap_cap]
    uint32_t *hist_out;   // optional [nspec * kHist]
    int32_t *err;         // device guard word
};

// ---- minHeap<hCell> of the reference (source/core/include/minheap.h:103-271) ------
__device__ __forceinline__ void heap_sift(Cell *a, int size, int i)
{
    for (;;) {
        const int r = (i + 1) * 2, l = r - 1;
        int s = i;
        float sv = a[i].h;
        if (l < size && a[l].h < sv) { s = l; sv = a[l].h; }
        if (r < size && a[r].h < sv) { s = r; }
        if (s == i) return;
        const Cell t = a[s];
        a[s] = a[i];
        a[i] = t;
        i = s;
    }
}

__device__ __forceinline__ void heap_insert(Cell *a, int &size, int cap, const Cell &c)
{
    if (size == cap) {
        if (c.h < a[0].h) return;
        a[0] = c;
        heap_sift(a, size, 0);
        return;
    }
    a[size++] = c;
    for (int i = (size - 1) / 2; i >= 0; i--) heap_sift(a, size, i);
}

// A spectrum gets an e-value when it has at least min_cpsm candidate PSMs and at least one
// (min_cpsm 0 acts as 1: with no candidate PSM the heap is empty and there is no top score).
__device__ __forceinline__ bool fits_tail(int32_t cpsms, uint32_t min_cpsm)
{
    return cpsms > 0 && (uint32_t)cpsms >= min_cpsm;
}

// The outputs of spectrum s when it is not searched (no probed bin, or a spectrum the
// device guard rejected): a zeroed result record with `status`, an empty histogram row
// and an empty heap row.  Called by every thread of the block (nthreads of them).
__device__ __forceinline__ void write_empty_row(const SearchArgs &a, uint32_t *hist, uint32_t s, int32_t status,
                                                int tid, int nthreads)
{
    if (tid == 0) {
        gx_result r;
        memset(&r, 0, sizeof(r));
        r.status = status;
        a.out[s] = r;
    }
    if (hist)
        for (int i = tid; i < kHist; i += nthreads) hist[(uint64_t)s * kHist + i] = 0u;
    if (a.heap_out)
        for (int i = tid; i < a.heap_cap; i += nthreads) a.heap_out[(uint64_t)s * a.heap_cap + i] = gx_cell{};
}

__device__ __forceinline__ Cell heap_getmax(const Cell *a, int size)
{
    if (size <= 1) return a[0];
    Cell m = a[size - 1];
    for (int k = size - 2; k >= size / 2; k--)
        if (a[k].h > m.h) m = a[k];
    return m;
}

// double -> int with x86-64 cvttsd2si semantics (INT_MIN for NaN / out of range).
__device__ __forceinline__ int32_t to_int_x86(double v)
{
    if (!(v > -2147483649.0 && v < 2147483648.0)) return (int32_t)0x80000000;
    return (int32_t)v;
}

// expeRT::ModelTailFit (source/core/expeRT.cpp:396-559) followed by the e-value of
// source/core/dslim_query.cpp:1017-1061.  Serial FP64 in one thread; the sums run in
// the reference's order so the fit matches it.  `sx` is scratch for kHist+1 doubles.
__device__ inline void tail_fit(const uint32_t *hist, int32_t cpsms, int32_t hyp, double *sx_buf, gx_result &r)
{
    double mu_t = 0.0, beta_t = 4.0;
    int end1 = hyp - 1;
    for (int p = hyp - 1; p >= 0; p--) if ((double)hist[p] >= 1.0) { end1 = p; break; }
    int stt1 = 0;
    for (int p = 0; p <= end1; p++) if ((double)hist[p] >= 1.0) { stt1 = p; break; }
    if (stt1 == end1) end1 += 1;
    if (cpsms < 1) {
        mu_t = 0.0;
        beta_t = 100.0;
    } else {
        sx_buf[0] = 0.0;  // the element before the slice (read when mark == -1)
        double *sx = sx_buf + 1;
        int size = end1 - stt1 + 1;
        if (size < 0) size = 0;
        double acc = 0.0;
        for (int i = 0; i < size; i++) { acc = acc + (double)hist[stt1 + i]; sx[i] = acc; }
        for (int i = 0; i < size; i++) {
            double v = sx[i] / (double)cpsms;
            v = v + (-1.0);
            sx[i] = -v;
            if (sx[i] > 1.0) sx[i] = 0.999;
        }
        if (size > 0) {
            int rep = size - 1;
            for (int p = size - 1; p >= 0; p--) if (sx[p] >= 1e-4) { rep = p; break; }
            const double v = sx[rep];
            for (int i = 0; i < size; i++) if (sx[i] <= 0.0) sx[i] = v;
        }
        for (int i = 0; i < size; i++) sx[i] = log10(sx[i]);
        int mark = 0, mark2 = 0;
        if (size >= 3) {
            const double hgt = sx[size - 1] - sx[0];
            const double t22 = sx[0] + hgt * 0.22;
            int lm = 0;
            for (int p = 0; p <= size - 1; p++) if (sx[p] <= t22) { lm = p; break; }
            mark = lm - 1;
            mark2 = size - 1;
            if (size > 3) {
                const double t87 = sx[0] + hgt * 0.87;
                for (int p = size - 1; p >= 0; p--) if (sx[p] >= t87) { mark2 = p; break; }
            }
            if (mark >= mark2) mark = mark2 - 1;
        } else {
            mark = 0;
            mark2 = size - 1;
        }
        const int n = mark2 - mark + 1;
        if (n == 1) {
            mu_t = 0.0;
            beta_t = sx[mark];
        } else if (n >= 2) {
            double xbar = 0.0, ybar = 0.0;
            for (int i = 0; i < n; i++) {
                xbar = xbar + (double)(stt1 + mark + i);
                ybar = ybar + sx[mark + i];
            }
            xbar = xbar / (double)n;
            ybar = ybar / (double)n;
            double top = 0.0, bot = 0.0;
            for (int i = 0; i < n; i++) {
                const double dx = (double)(stt1 + mark + i) - xbar;
                top = top + dx * (sx[mark + i] - ybar);
                bot = bot + dx * dx;
            }
            mu_t = top / bot;
            beta_t = ybar - mu_t * xbar;
        } else {
            mu_t = __longlong_as_double(0x7ff8000000000000ll);
            beta_t = mu_t;
        }
    }
    r.slope = mu_t;
    r.icpt = beta_t;
    r.mu = to_int_x86(mu_t * 1e6);
    r.beta = to_int_x86(beta_t * 1e6);
    r.stt1 = stt1;
    r.end1 = end1;
    double w = (double)r.mu, b = (double)r.beta;
    w /= 1e6;
    b /= 1e6;
    const double lgs = (w * (double)hyp) + b;
    r.e_x = pow(10.0, lgs) * (double)(uint32_t)cpsms;
    r.e_fp64 = pow(10.0, mu_t * (double)hyp + beta_t) * (double)(uint32_t)cpsms;
}


// tail_fit with its elementwise steps, integer prefix sums and searches spread over a warp.
// Bit-identical to tail_fit: prefix sums of integer counts are exact in FP64, every other
// parallel step is elementwise or a search, and the order-dependent least-squares sums stay
// in lane 0.  All 32 lanes call it; lane 0 fills r.
__device__ inline void tail_fit_warp(const uint32_t *hist, int32_t cpsms, int32_t hyp, double *sx_buf, gx_result &r,
                                     int lane)
{
    constexpr unsigned kAll = 0xffffffffu;
    constexpr int kNone = 0x7fffffff;
    int e = -1;
    for (int p = hyp - 1 - lane; p >= 0; p -= 32)
        if (hist[p] >= 1u) { e = p; break; }
    for (int o = 16; o; o >>= 1) e = max(e, __shfl_xor_sync(kAll, e, o));
    int end1 = e >= 0 ? e : hyp - 1;
    int st = kNone;
    for (int p = lane; p <= end1; p += 32)
        if (hist[p] >= 1u) { st = p; break; }
    for (int o = 16; o; o >>= 1) st = min(st, __shfl_xor_sync(kAll, st, o));
    const int stt1 = st == kNone ? 0 : st;
    if (stt1 == end1) end1 += 1;
    double mu_t = 0.0, beta_t = 4.0;
    if (cpsms < 1) {
        mu_t = 0.0;
        beta_t = 100.0;
    } else {
        if (lane == 0) sx_buf[0] = 0.0;  // the element before the slice (read when mark == -1)
        double *sx = sx_buf + 1;
        const int size = max(0, end1 - stt1 + 1);
        // cumulative counts: lane l sums a contiguous run, then a warp scan
        const int per = (size + 31) / 32;
        const int b0 = min(size, lane * per), b1 = min(size, b0 + per);
        unsigned long long part = 0;
        for (int i = b0; i < b1; i++) part += hist[stt1 + i];
        unsigned long long incl = part;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(kAll, incl, o);
            if (lane >= o) incl += y;
        }
        unsigned long long run = incl - part;
        for (int i = b0; i < b1; i++) {
            run += hist[stt1 + i];
            sx[i] = (double)run;
        }
        __syncwarp();
        for (int i = lane; i < size; i += 32) {
            double v = sx[i] / (double)cpsms;
            v = v + (-1.0);
            sx[i] = -v;
            if (sx[i] > 1.0) sx[i] = 0.999;
        }
        __syncwarp();
        if (size > 0) {
            int rp = -1;
            for (int p = size - 1 - lane; p >= 0; p -= 32)
                if (sx[p] >= 1e-4) { rp = p; break; }
            for (int o = 16; o; o >>= 1) rp = max(rp, __shfl_xor_sync(kAll, rp, o));
            const double v = sx[rp >= 0 ? rp : size - 1];
            __syncwarp();
            for (int i = lane; i < size; i += 32)
                if (sx[i] <= 0.0) sx[i] = v;
        }
        __syncwarp();
        for (int i = lane; i < size; i += 32) sx[i] = log10(sx[i]);
        __syncwarp();
        int mark = 0, mark2 = 0;
        if (size >= 3) {
            const double hgt = sx[size - 1] - sx[0];
            const double t22 = sx[0] + hgt * 0.22;
            int lm = kNone;
            for (int p = lane; p < size; p += 32)
                if (sx[p] <= t22) { lm = p; break; }
            for (int o = 16; o; o >>= 1) lm = min(lm, __shfl_xor_sync(kAll, lm, o));
            mark = (lm == kNone ? 0 : lm) - 1;
            mark2 = size - 1;
            if (size > 3) {
                const double t87 = sx[0] + hgt * 0.87;
                int m2 = -1;
                for (int p = size - 1 - lane; p >= 0; p -= 32)
                    if (sx[p] >= t87) { m2 = p; break; }
                for (int o = 16; o; o >>= 1) m2 = max(m2, __shfl_xor_sync(kAll, m2, o));
                if (m2 >= 0) mark2 = m2;
            }
            if (mark >= mark2) mark = mark2 - 1;
        } else {
            mark = 0;
            mark2 = size - 1;
        }
        const int n = mark2 - mark + 1;
        if (lane == 0) {
            if (n == 1) {
                mu_t = 0.0;
                beta_t = sx[mark];
            } else if (n >= 2) {
                double xbar = 0.0, ybar = 0.0;
                for (int i = 0; i < n; i++) {
                    xbar = xbar + (double)(stt1 + mark + i);
                    ybar = ybar + sx[mark + i];
                }
                xbar = xbar / (double)n;
                ybar = ybar / (double)n;
                double top = 0.0, bot = 0.0;
                for (int i = 0; i < n; i++) {
                    const double dx = (double)(stt1 + mark + i) - xbar;
                    top = top + dx * (sx[mark + i] - ybar);
                    bot = bot + dx * dx;
                }
                mu_t = top / bot;
                beta_t = ybar - mu_t * xbar;
            } else {
                mu_t = __longlong_as_double(0x7ff8000000000000ll);
                beta_t = mu_t;
            }
        }
    }
    if (lane == 0) {
        r.slope = mu_t;
        r.icpt = beta_t;
        r.mu = to_int_x86(mu_t * 1e6);
        r.beta = to_int_x86(beta_t * 1e6);
        r.stt1 = stt1;
        r.end1 = end1;
        double w = (double)r.mu, b = (double)r.beta;
        w /= 1e6;
        b /= 1e6;
        const double lgs = (w * (double)hyp) + b;
        r.e_x = pow(10.0, lgs) * (double)(uint32_t)cpsms;
        r.e_fp64 = pow(10.0, mu_t * (double)hyp + beta_t) * (double)(uint32_t)cpsms;
    }
}

}  // namespace gx
