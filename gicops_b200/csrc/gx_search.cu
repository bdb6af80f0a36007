// Query path on sm_100a: precursor windows, fragment-ion bucket probes into a shared-
// memory BYC scorecard, hyperscore + histogram + exact top-K heap, FP64 tail fit.
//
// Reference behaviour followed (paths relative to the reference project):
//   source/core/dslim_query.cpp:749-1242 (DSLIM_QuerySpectrum, DSLIM_BinarySearch)
//   source/core/expeRT.cpp:396-559, 1149-1289 (ModelTailFit, LinearFit)
//   source/core/include/minheap.h:103-271 (top-K heap)
// Compiled with -fmad=false: no multiply-add is fused, so every FP64 step rounds as
// the reference's x86-64 build does.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/gicops_b200.h"
#include "gx_batched.h"
#include "gx_device_scope.cuh"
#include "gx_index.cuh"
#include "gx_device.cuh"
#include "gx_internal.h"

namespace gx {

namespace {
thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0};
}  // namespace

gx_status fail(gx_status code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

namespace {
thread_local bool t_capturing = false;   // kernels issued into a graph capture are counted per replay
}
void count_launch(uint64_t n)
{
    if (!t_capturing) g_launches.fetch_add(n, std::memory_order_relaxed);
}

// ---- opt-in kernel timing --------------------------------------------------------------
namespace {
struct ProfRec {
    const char *name;
    cudaEvent_t a, b;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRec> g_prof;
}  // namespace

// Records a start event on `st` when timing is on; returns a handle for prof_end.
int prof_begin(const char *name, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (!g_prof_on) return -1;
    ProfRec r{name, nullptr, nullptr};
    if (cudaEventCreate(&r.a) != cudaSuccess || cudaEventCreate(&r.b) != cudaSuccess) return -1;
    cudaEventRecord(r.a, st);
    std::lock_guard<std::mutex> g(g_prof_mu);
    g_prof.push_back(r);
    return (int)g_prof.size() - 1;
}

void prof_end(int h, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (h < 0) return;
    std::lock_guard<std::mutex> g(g_prof_mu);
    if (h < (int)g_prof.size()) cudaEventRecord(g_prof[h].b, st);
}

gx_status cuda_fail(int e, const char *what)
{
    return fail(GX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString((cudaError_t)e));
}

#define GX_CUDA(call)                                       \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// ------------------------------------------------------------------------------------
// Kernels
// ------------------------------------------------------------------------------------

// Window [lo, hi] of every (spectrum, length): first entry with mass >= prec-dM, last
// with mass <= prec+dM, both bounds rounded to float as the reference does
// (dslim_query.cpp:1102-1164; its bisection helpers compute lower/upper bounds).
__global__ void k_windows(SearchArgs a, int2 *win)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)a.nspec * a.nlen) return;
    const uint32_t s = (uint32_t)(i / a.nlen);
    const int l = (int)(i - (uint64_t)s * a.nlen);
    const DevLen ln = a.lens[l];
    const double dM = a.dMq ? a.dMq[s] : a.dM;
    int lo = 1, hi = 0;
    if (!(dM < 0.0) && ln.npep > 0) {
        const float pr = a.prec[s];
        const float p1 = __double2float_rn(__dsub_rn((double)pr, dM));
        const float p2 = __double2float_rn(__dadd_rn((double)pr, dM));
        const float *m = a.mass + ln.mass_off;
        const uint32_t N = ln.npep;
        if (p1 == p1 && p2 == p2 && !(p1 > m[N - 1]) && !(p2 < m[0])) {
            uint32_t x = 0, y = N;
            while (x < y) {
                const uint32_t c = (x + y) >> 1;
                if (m[c] < p1) x = c + 1; else y = c;
            }
            lo = (int)x;
            x = 0;
            y = N;
            while (x < y) {
                const uint32_t c = (x + y) >> 1;
                if (p2 < m[c]) y = c; else x = c + 1;
            }
            hi = (int)x - 1;
        }
    }
    win[i] = make_int2(lo, hi);
}

__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *__restrict__ v, uint32_t a, uint32_t b,
                                                    uint32_t key)
{
    while (a < b) {
        const uint32_t c = a + ((b - a) >> 1);
        if (__ldg(v + c) < key) a = c + 1; else b = c;
    }
    return a;
}

constexpr int kBlock = 512;
constexpr int kWarps = kBlock / 32;

struct SearchSmem {
    int32_t qmz[GX_MAX_PEAKS];
    uint32_t qin[GX_MAX_PEAKS];
    uint32_t hist[kHist];
    double lgf[81];
    Cell heap[kMaxHeap + 1];
    Cell ent[kBlock];
    int32_t warp_cnt[kWarps];
    int32_t npk;
    int32_t heap_size;
    int32_t cpsms;
    int32_t nent;
    int32_t wide;
    int32_t status;
    float root;
};

// Scorecard words.  Packed (8 B per candidate): low word b ions, high word y ions,
// each [count:8 | intensity sum:24]; valid while every per-candidate count stays
// below 256 and every intensity sum below 2^24 (checked per spectrum).  Wide (12 B
// per candidate): u32 counts (b low 16, y high 16), u32 b sum, u32 y sum, with the
// reference's uint wrap-around.
__device__ __forceinline__ void card_add_packed(unsigned long long *sc, uint32_t c, uint32_t isY, uint32_t in)
{
    const unsigned long long v = (unsigned long long)((1u << 24) | in) << (isY ? 32 : 0);
    atomicAdd(sc + c, v);
}

// One spectrum per CTA.  Lengths run in index order, each window in tiles of
// `tile` candidates; a tile is filled by probing every (peak, bin) bucket for the
// ion ids whose entry falls in the tile, then scanned in entry order.
__global__ void __launch_bounds__(kBlock) k_search_plain(SearchArgs a, int tile)
{
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ SearchSmem sm;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint32_t s = blockIdx.x;
    if (s >= a.nspec) return;

    // ---- peaks (only those the reference probes) -----------------------------------
    if (tid == 0) {
        sm.npk = 0;
        sm.heap_size = 0;
        sm.cpsms = 0;
        sm.status = 0;
        sm.root = 0.0f;
    }
    for (int i = tid; i < kHist; i += kBlock) sm.hist[i] = 0;
    for (int i = tid; i < 81; i += kBlock) sm.lgf[i] = a.lgfact[i];
    __syncthreads();
    const uint32_t q0 = a.qidx[s], q1 = a.qidx[s + 1];
    if (q1 < q0 || q1 - q0 > GX_MAX_PEAKS) {   // not searched: a defined row, flagged
        if (tid == 0) atomicExch(a.err, 1);
        write_empty_row(a, a.hist_out, s, GX_STATUS_PEAK_LIMIT, tid, kBlock);
        return;
    }
    unsigned long long sum_in = 0;
    for (uint32_t k = q0 + tid; k < q1; k += kBlock) {
        const int32_t qi = a.moz[k];
        if (qi > (int32_t)a.dF && (double)qi < a.upper) {
            const int slot = atomicAdd(&sm.npk, 1);
            sm.qmz[slot] = qi;
            sm.qin[slot] = (uint32_t)a.intn[k];
            sum_in += (uint32_t)a.intn[k];
        }
    }
    // block sum of intensities for the packed-scorecard guard
    for (int o = 16; o; o >>= 1) sum_in += __shfl_xor_sync(0xffffffffu, sum_in, o);
    __shared__ unsigned long long wsum[kWarps];
    if (lane == 0) wsum[wid] = sum_in;
    __syncthreads();
    if (tid == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kWarps; w++) t += wsum[w];
        const bool ok = (uint64_t)sm.npk * a.maxz <= 255u && t * a.maxz < (1ull << 24);
        sm.wide = (!ok || (a.flags & GX_FLAG_WIDE_SCORECARD)) ? 1 : 0;
        if (sm.wide) sm.status |= 8;
    }
    __syncthreads();
    // Peaks must be probed in any order: the scorecard sums are integer.
    const int npk = sm.npk;
    const bool wide = sm.wide != 0;
    const int W = 2 * (int)a.dF + 1;
    const int ctile = wide ? (tile * 2) / 3 : tile;
    unsigned long long *scp = reinterpret_cast<unsigned long long *>(dyn);
    uint32_t *scw_cnt = reinterpret_cast<uint32_t *>(dyn);
    uint32_t *scw_ib = scw_cnt + ctile;
    uint32_t *scw_iy = scw_ib + ctile;
    for (int i = tid; i < (wide ? 3 * ctile : 2 * ctile); i += kBlock) reinterpret_cast<uint32_t *>(dyn)[i] = 0;
    __syncthreads();

    for (int ixx = 0; ixx < a.nlen; ixx++) {
        const int2 w = a.win[(uint64_t)s * a.nlen + ixx];
        if (w.y < w.x) continue;
        const DevLen ln = a.lens[ixx];
        const uint32_t *__restrict__ bA = a.bA + (uint64_t)ixx * a.nbins;
        const uint32_t *__restrict__ iA = a.iA + ln.ia_off;
        const uint32_t speclen = ln.speclen;
        for (int t0 = w.x; t0 <= w.y; t0 += ctile) {
            const int t1 = min(w.y + 1, t0 + ctile);
            const int tn = t1 - t0;
            // device ids are 2*entry + (y ion): the tile is [2*t0, 2*t1)
            const uint32_t idlo = 2u * (uint32_t)t0, idhi = 2u * (uint32_t)t1;
            // ---- probe buckets, scatter into the scorecard ----------------------------
            for (int it = tid; it < npk * W; it += kBlock) {
                const int k = it / W;
                const uint32_t bin = (uint32_t)(sm.qmz[k] - (int32_t)a.dF + (it - k * W));
                const uint32_t b0 = __ldg(bA + bin), b1 = __ldg(bA + bin + 1);
                if (b1 <= b0) continue;
                const uint32_t x = lower_bound_u32(iA, b0, b1, idlo);
                const uint32_t y = lower_bound_u32(iA, x, b1, idhi);
                const uint32_t in = sm.qin[k];
                for (uint32_t ion = x; ion < y; ion++) {
                    const uint32_t raw = __ldg(iA + ion);
                    const uint32_t isY = raw & 1u;
                    const uint32_t c = (raw >> 1) - (uint32_t)t0;
                    if (!wide) {
                        card_add_packed(scp, c, isY, in);
                    } else {
                        atomicAdd(scw_cnt + c, isY ? 0x10000u : 1u);
                        atomicAdd((isY ? scw_iy : scw_ib) + c, in);
                    }
                }
            }
            __syncthreads();
            // ---- scan the tile in entry order ---------------------------------------
            for (int c0 = 0; c0 < tn; c0 += kBlock) {
                const int c = c0 + tid;
                bool psm = false;
                Cell cell;
                if (c < tn) {
                    uint32_t bc, yc, ib, iy;
                    if (!wide) {
                        const unsigned long long v = scp[c];
                        const uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
                        bc = lo >> 24; ib = lo & 0xFFFFFFu; yc = hi >> 24; iy = hi & 0xFFFFFFu;
                        scp[c] = 0ull;
                    } else {
                        const uint32_t cnt = scw_cnt[c];
                        bc = cnt & 0xFFFFu; yc = cnt >> 16; ib = scw_ib[c]; iy = scw_iy[c];
                        scw_cnt[c] = 0; scw_ib[c] = 0; scw_iy[c] = 0;
                    }
                    const uint32_t shpk = (bc + yc) & 0xFFFFu;
                    if (shpk >= a.min_shp) {
                        uint32_t bi = bc, yi = yc;
                        if (bi > 80u || yi > 80u) {
                            atomicOr(&sm.status, 4);
                            bi = min(bi, 80u);
                            yi = min(yi, 80u);
                        }
                        const double h1 = sm.lgf[bi] + sm.lgf[yi];
                        float h = __double2float_rn(h1 + log10((double)(uint32_t)(1u + ib)) +
                                                    log10((double)(uint32_t)(1u + iy)) - 4.0);
                        if (h > 0.0f) {
                            if (h >= 80.0f) h = 79.0f;
                            psm = true;
                            cell.h = h;
                            cell.psid = t0 + c;
                            cell.ixx = (uint16_t)ixx;
                            cell.shp = (uint16_t)shpk;
                            cell.total = (uint16_t)speclen;
                            cell.pad = 0;
                            const int hb = __double2int_rz(__dadd_rn((double)__fmul_rn(h, 10.0f), 0.5));
                            atomicAdd(&sm.hist[hb], 1u);
                        }
                    }
                }
                // entrants of the exact heap: every PSM while it is not full, else h >= root
                const bool ent = psm && (sm.heap_size < a.heap_cap || cell.h >= sm.root);
                const unsigned bal = __ballot_sync(0xffffffffu, ent);
                const unsigned pbal = __ballot_sync(0xffffffffu, psm);
                if (lane == 0) sm.warp_cnt[wid] = __popc(bal);
                if (lane == 0 && pbal) atomicAdd(&sm.cpsms, __popc(pbal));
                __syncthreads();
                if (ent) {
                    int base = 0;
                    for (int w2 = 0; w2 < wid; w2++) base += sm.warp_cnt[w2];
                    sm.ent[base + __popc(bal & ((1u << lane) - 1u))] = cell;
                }
                __syncthreads();
                if (tid == 0) {
                    int ne = 0;
                    for (int w2 = 0; w2 < kWarps; w2++) ne += sm.warp_cnt[w2];
                    int hs = sm.heap_size;
                    for (int e = 0; e < ne; e++) heap_insert(sm.heap, hs, a.heap_cap, sm.ent[e]);
                    sm.heap_size = hs;
                    sm.root = sm.heap[0].h;
                }
                __syncthreads();
            }
        }
    }

    // ---- epilogue: top PSM, tail fit, outputs -----------------------------------------
    if (a.hist_out)
        for (int i = tid; i < kHist; i += kBlock) a.hist_out[(uint64_t)s * kHist + i] = sm.hist[i];
    if (a.heap_out)
        for (int i = tid; i < a.heap_cap; i += kBlock) {
            gx_cell o{};
            if (i < sm.heap_size) {
                const Cell c = sm.heap[i];
                o.hyperscore = c.h; o.psid = c.psid; o.idxoffset = c.ixx; o.sharedions = c.shp; o.totalions = c.total;
            }
            a.heap_out[(uint64_t)s * a.heap_cap + i] = o;
        }
    if (tid == 0) {
        gx_result r;
        memset(&r, 0, sizeof(r));
        r.cpsms = sm.cpsms;
        int st = sm.status;
        if (fits_tail(sm.cpsms, a.min_cpsm)) {
            st |= 1;
            const Cell t = heap_getmax(sm.heap, sm.heap_size);
            r.top.hyperscore = t.h; r.top.psid = t.psid; r.top.idxoffset = t.ixx;
            r.top.sharedions = t.shp; r.top.totalions = t.total;
            r.maxhyp = __double2int_rz(__dadd_rn((double)__fmul_rn(t.h, 10.0f), 0.5));
            tail_fit(sm.hist, sm.cpsms, r.maxhyp, reinterpret_cast<double *>(dyn), r);
            if (r.e_x < a.expect_max) st |= 2;
        }
        r.status = st;
        a.out[s] = r;
    }
}

}  // namespace gx

// ------------------------------------------------------------------------------------
// Host API
// ------------------------------------------------------------------------------------
using namespace gx;

namespace {
constexpr int kDefaultTile = 8192;   // plain path: candidates per scorecard tile (8 B each)
}

struct gx_workspace {
    const gx_index *ix = nullptr;
    int device = 0;   // the index's device (the index may be freed first)
    uint32_t max_spec = 0, max_peaks = 0;
    int2 *win = nullptr;
    double *lgfact = nullptr;
    int32_t *err = nullptr;
    // learned tail applied after the tail fit (batched path), when attached
    gx_tail_model *tail = nullptr;
    uint32_t tail_below = 0;
    // staging for gx_search_host
    uint32_t *qidx = nullptr;
    int32_t *moz = nullptr, *intn = nullptr, *charge = nullptr;
    float *prec = nullptr;
    double *dMq = nullptr;
    gx_result *out = nullptr;
    gx_cell *heap = nullptr;
    uint32_t *hist = nullptr;
    cudaStream_t stream = nullptr;
    // batched path
    Interval *ivl = nullptr;
    uint32_t *nivl = nullptr, *guard = nullptr, *queue = nullptr, *hist_g = nullptr;
    Cell *spill = nullptr;
    uint32_t spill_per_warp = 0;
    double *logtab = nullptr;
    BatchedScratch bs{};
    int tile = kBlockEntries;   // largest candidate tile the buffers hold (the index's block)
    BatchedTiles tiles{};       // launch shape of the batched path (gx_workspace_set_tiles, gx_autotune)
    // CUDA graphs of the batched launch sequence (gx_workspace_set_graph): one per key of
    // buffers, parameters, shape and attached tail, the most recent kGraphs kept
    bool graph_on = false;
    struct Graph {
        std::vector<unsigned char> key;
        cudaGraphExec_t exec = nullptr;
        uint64_t kernels = 0;
    };
    std::vector<Graph> graphs;
    cudaEvent_t gev_in = nullptr, gev_out = nullptr;
};

extern "C" const char *gx_last_error(void) { return g_last_error.c_str(); }

extern "C" gx_status gx_profile_enable(int32_t on)
{
    std::lock_guard<std::mutex> g(g_prof_mu);
    for (auto &r : g_prof) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    g_prof.clear();
    g_prof_on = on != 0;
    return GX_SUCCESS;
}

extern "C" int32_t gx_profile_read(gx_kernel_time *out, int32_t cap)
{
    std::lock_guard<std::mutex> g(g_prof_mu);
    std::vector<gx_kernel_time> agg;
    for (auto &r : g_prof) {
        float ms = 0.0f;
        if (cudaEventSynchronize(r.b) != cudaSuccess || cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) continue;
        gx_kernel_time *t = nullptr;
        for (auto &x : agg)
            if (std::strncmp(x.name, r.name, sizeof(x.name)) == 0) t = &x;
        if (!t) {
            agg.push_back(gx_kernel_time{});
            t = &agg.back();
            std::strncpy(t->name, r.name, sizeof(t->name) - 1);
        }
        t->launches += 1;
        t->total_ms += ms;
    }
    const int n = (int)agg.size();
    for (int i = 0; i < n && i < cap; i++) out[i] = agg[i];
    return n;
}
extern "C" uint64_t gx_launch_count(void) { return g_launches.load(); }

extern "C" void gx_lgfact(double *o)
{
    o[0] = o[1] = std::log10(1.0);
    for (int i = 2; i < 81; i++) o[i] = std::log10((double)i) + o[i - 1];
}

extern "C" int32_t gx_heap_capacity(uint32_t topmatches)
{
    uint32_t num = topmatches == 0 ? 1 : topmatches;
    num = (uint32_t)(std::floor(std::log2((double)num) + 0.999));
    return (int32_t)((1u << num) - 1u);
}



extern "C" gx_status gx_workspace_free(gx_workspace *ws)
{
    if (!ws) return GX_SUCCESS;
    DeviceScope ds(ws->device);
    void *ptrs[] = {ws->win, ws->lgfact, ws->err, ws->qidx, ws->moz, ws->intn, ws->charge, ws->prec,
                    ws->dMq, ws->out, ws->heap, ws->hist, ws->ivl, ws->nivl, ws->guard, ws->queue,
                    ws->hist_g, ws->spill, ws->logtab, ws->bs.key_in, ws->bs.key_out, ws->bs.ord_in, ws->bs.ord_out, ws->bs.sort_temp};
    for (void *p : ptrs) cudaFree(p);
    for (auto &g : ws->graphs) cudaGraphExecDestroy(g.exec);
    if (ws->gev_in) cudaEventDestroy(ws->gev_in);
    if (ws->gev_out) cudaEventDestroy(ws->gev_out);
    if (ws->stream) cudaStreamDestroy(ws->stream);
    delete ws;
    cudaGetLastError();   // nothing of a free is reported to the next call
    return GX_SUCCESS;
}

extern "C" gx_status gx_workspace_create(const gx_index *ix, uint32_t max_spec, uint32_t max_peaks,
                                         gx_workspace **out)
{
    if (!ix || !out) return fail(GX_ERR_INVLD_PTR, "gx_workspace_create: null argument");
    *out = nullptr;
    if (max_spec == 0) return fail(GX_ERR_INVLD_PARAM, "gx_workspace_create: max_spec must be > 0");
    DeviceScope ds(ix->device);
    GX_CUDA(ds.status());
    auto *ws = new gx_workspace();
    ws->ix = ix;
    ws->device = ix->device;
    ws->max_spec = max_spec;
    ws->max_peaks = max_peaks;
    cudaError_t e = cudaSuccess;
    const uint64_t nw = (uint64_t)max_spec * ix->nlen;
    auto al = [&](void **p, uint64_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes ? bytes : 16);
    };
    al((void **)&ws->win, sizeof(int2) * nw);
    al((void **)&ws->lgfact, sizeof(double) * 81);
    al((void **)&ws->err, sizeof(int32_t));
    al((void **)&ws->qidx, sizeof(uint32_t) * (max_spec + 1));
    al((void **)&ws->moz, sizeof(int32_t) * (uint64_t)max_peaks);
    al((void **)&ws->intn, sizeof(int32_t) * (uint64_t)max_peaks);
    al((void **)&ws->charge, sizeof(int32_t) * max_spec);
    al((void **)&ws->prec, sizeof(float) * max_spec);
    al((void **)&ws->dMq, sizeof(double) * max_spec);
    al((void **)&ws->out, sizeof(gx_result) * max_spec);
    al((void **)&ws->ivl, sizeof(Interval) * 2 * (uint64_t)(max_peaks ? max_peaks : 1));
    al((void **)&ws->nivl, sizeof(uint32_t) * max_spec);
    al((void **)&ws->guard, sizeof(uint32_t) * max_spec);
    al((void **)&ws->queue, 2 * sizeof(uint32_t));
    al((void **)&ws->hist_g, sizeof(uint32_t) * GX_HIST_BINS * (uint64_t)max_spec);
    al((void **)&ws->bs.key_in, sizeof(uint64_t) * max_spec);
    al((void **)&ws->bs.key_out, sizeof(uint64_t) * max_spec);
    al((void **)&ws->bs.ord_in, sizeof(uint32_t) * max_spec);
    al((void **)&ws->bs.ord_out, sizeof(uint32_t) * max_spec);
    ws->bs.sort_temp_bytes = batched_sort_temp_bytes(max_spec);
    al(&ws->bs.sort_temp, ws->bs.sort_temp_bytes);
    if (e == cudaSuccess) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = batched_set_attributes(ws->tile);
        ws->bs.sms = sms;
        for (int c = 1; c <= 3; c++) {
            ws->bs.max_ctas[c] = batched_ctas_per_sm(ws->tile, c);
            ws->bs.piped_ok[c] = piped_fits(ws->tile, c);
        }
    }
    ws->tiles.tile = ws->tile;
    ws->spill_per_warp = batched_spill_per_warp(ws->tile);
    // entrant spill of every warp of the largest grid (two CTAs of 16 warps per SM)
    al((void **)&ws->spill, sizeof(Cell) * (uint64_t)ws->bs.sms * 32 * ws->spill_per_warp);
    al((void **)&ws->logtab, sizeof(double) * kLogTab);
    if (e == cudaSuccess) e = fill_logtab(ws->logtab, kLogTab, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = batched_set_attributes(ws->tile);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        cudaGetLastError();
        gx_workspace_free(ws);
        return fail(GX_ERR_BAD_MEM_ALLOC, std::string("gx_workspace_create: ") + cudaGetErrorString(e));
    }
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_search_plain, cudaFuncAttributeMaxDynamicSharedMemorySize, kDefaultTile * 8);
    if (e != cudaSuccess) {
        gx_workspace_free(ws);
        return cuda_fail(e, "gx_workspace_create: kernel attributes");
    }
    double lg[81];
    gx_lgfact(lg);
    if ((e = cudaMemcpy(ws->lgfact, lg, sizeof(lg), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(ws->err, 0, sizeof(int32_t))) != cudaSuccess) {
        gx_workspace_free(ws);
        return cuda_fail(e, "gx_workspace_create");
    }
    *out = ws;
    return GX_SUCCESS;
}

namespace {

gx_status check_params(const gx_index *ix, const gx_params *p, int32_t *cap)
{
    *cap = gx_heap_capacity(p->topmatches);
    if (*cap < 1 || *cap > GX_MAX_HEAP)
        return fail(GX_ERR_INVLD_PARAM, "topmatches gives a top-K heap capacity outside 1..31");
    if (p->scale == 0 || p->dF > 255 || p->min_shp == 0)
        return fail(GX_ERR_INVLD_PARAM, "scale must be > 0, dF <= 255, min_shp >= 1");
    // bins probed: up to (max_mass*scale - 1 - dF) + dF + 1 must stay inside bA
    const double top = p->max_mass * (double)p->scale;
    if (!(top >= 1.0) || top + 1.0 > (double)ix->nbins + 0.5)
        return fail(GX_ERR_INVLD_PARAM, "max_mass*scale+1 must not exceed the index's bins");
    // the packed scorecard needs at most one ion per (charge, series) in a fragment window
    if ((2.0 * p->dF + 1.0) * ix->maxz >= 57.02 * p->scale)
        return fail(GX_ERR_INVLD_PARAM, "fragment tolerance wider than the smallest residue");
    return GX_SUCCESS;
}

gx_status launch_direct(gx_index *ix, gx_workspace *ws, const gx_queries *q, const gx_params *p, gx_result *out,
                        gx_cell *heap, uint32_t *hist, cudaStream_t st)
{
    int32_t cap;
    gx_status rc = check_params(ix, p, &cap);
    if (rc != GX_SUCCESS) return rc;
    cudaGetLastError();   // an earlier call's error is not ours to report
    if (q->nspec > ws->max_spec) return fail(GX_ERR_INVLD_SIZE, "more spectra than the workspace holds");
    if (q->nspec == 0) return GX_SUCCESS;
    SearchArgs a{};
    a.bA = ix->bA; a.iA = ix->iA; a.iAb = ix->iAb; a.blkA = ix->blkA; a.block = ix->block;
    a.iab_bytes = ix->iab_bytes; a.mass = ix->mass; a.lens = ix->lens; a.nlen = ix->nlen; a.nbins = ix->nbins;
    a.maxz = ix->maxz;
    a.qidx = q->idx; a.moz = q->moz; a.intn = q->intn; a.prec = q->prec; a.dMq = q->dM; a.nspec = q->nspec;
    a.dM = p->dM;
    a.upper = (p->max_mass * (double)p->scale) - 1.0 - (double)p->dF;
    a.dF = p->dF; a.min_shp = p->min_shp; a.min_cpsm = p->min_cpsm; a.heap_cap = cap;
    a.expect_max = p->expect_max; a.flags = p->flags; a.lgfact = ws->lgfact;
    a.win = ws->win; a.out = out; a.heap_out = heap; a.hist_out = hist; a.err = ws->err;

    if (!(p->flags & GX_FLAG_PLAIN)) {
        if (q->npeaks > ws->max_peaks) return fail(GX_ERR_INVLD_SIZE, "more peaks than the workspace holds");
        a.ivl = ws->ivl; a.ivl_cap = 2ull * ws->max_peaks; a.nivl = ws->nivl; a.guard = ws->guard; a.queue = ws->queue;
        a.hist_g = hist ? hist : ws->hist_g;
        a.spill = ws->spill;
        a.logtab = ws->logtab;
        a.logtab_n = kLogTab;
        a.spill_per_warp = ws->spill_per_warp;
        cudaError_t e = launch_batched(a, ws->bs, ws->tiles, st);
        if (e != cudaSuccess) return cuda_fail(e, "batched search launch");
        if (ws->tail && ws->tail_below)
            return gx_tail_apply(ws->tail, a.hist_g, out, q->prec, q->charge, q->nspec, ws->tail_below, p->expect_max,
                                 st);
        return GX_SUCCESS;
    }
    const uint64_t nw = (uint64_t)q->nspec * ix->nlen;
    int h = prof_begin("k_windows", st);
    k_windows<<<(unsigned)((nw + 255) / 256), 256, 0, st>>>(a, ws->win);
    prof_end(h, st);
    count_launch();
    const int tile = kDefaultTile;
    const size_t smem = (size_t)tile * 8;
    h = prof_begin("k_search_plain", st);
    k_search_plain<<<q->nspec, kBlock, smem, st>>>(a, tile);
    prof_end(h, st);
    count_launch();
    GX_CUDA(cudaGetLastError());
    return GX_SUCCESS;
}

constexpr size_t kGraphs = 4;

// Kernel nodes of a graph (for the launch count of its replays).
uint64_t kernel_nodes(cudaGraph_t g)
{
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return 0;
    std::vector<cudaGraphNode_t> nodes(n);
    if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
    uint64_t k = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
    }
    return k;
}

// The batched path's launch sequence through a CUDA graph: captured on the workspace's
// stream the first time a key (queries, parameters, outputs, launch shape, attached tail)
// is seen, replayed afterwards; ordered after the caller's earlier work on `st` and before
// its later work by two events.  The plain path and timed runs (gx_profile_enable) launch
// directly.
gx_status launch_search(gx_index *ix, gx_workspace *ws, const gx_queries *q, const gx_params *p, gx_result *out,
                        gx_cell *heap, uint32_t *hist, cudaStream_t st)
{
    if (!ws->graph_on || (p->flags & GX_FLAG_PLAIN) || g_prof_on || q->nspec == 0)
        return launch_direct(ix, ws, q, p, out, heap, hist, st);
    int32_t cap;
    gx_status rc = check_params(ix, p, &cap);   // refused before any capture
    if (rc != GX_SUCCESS) return rc;
    if (q->nspec > ws->max_spec || q->npeaks > ws->max_peaks)
        return fail(GX_ERR_INVLD_SIZE, "more spectra or peaks than the workspace holds");
    std::vector<unsigned char> key(sizeof(gx_queries) + sizeof(gx_params) + 3 * sizeof(void *) +
                                   sizeof(BatchedTiles) + sizeof(void *) + sizeof(uint32_t));
    unsigned char *k = key.data();
    auto put = [&](const void *v, size_t n) {
        std::memcpy(k, v, n);
        k += n;
    };
    put(q, sizeof(gx_queries));
    put(p, sizeof(gx_params));
    put(&out, sizeof(void *));
    put(&heap, sizeof(void *));
    put(&hist, sizeof(void *));
    put(&ws->tiles, sizeof(BatchedTiles));
    put(&ws->tail, sizeof(void *));
    put(&ws->tail_below, sizeof(uint32_t));
    cudaStream_t gs = ws->stream;
    gx_workspace::Graph *g = nullptr;
    for (auto &x : ws->graphs)
        if (x.key == key) g = &x;
    if (!g) {
        cudaGetLastError();
        GX_CUDA(cudaStreamBeginCapture(gs, cudaStreamCaptureModeThreadLocal));
        t_capturing = true;
        rc = launch_direct(ix, ws, q, p, out, heap, hist, gs);
        t_capturing = false;
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(gs, &graph);
        if (rc != GX_SUCCESS || e != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            return rc != GX_SUCCESS ? rc : cuda_fail(e, "search graph capture");
        }
        gx_workspace::Graph ng;
        ng.key = std::move(key);
        ng.kernels = kernel_nodes(graph);
        const cudaError_t ei = cudaGraphInstantiate(&ng.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) return cuda_fail(ei, "search graph instantiate");
        if (ws->graphs.size() >= kGraphs) {
            cudaGraphExecDestroy(ws->graphs.front().exec);
            ws->graphs.erase(ws->graphs.begin());
        }
        ws->graphs.push_back(std::move(ng));
        g = &ws->graphs.back();
    }
    if (st != gs) {
        GX_CUDA(cudaEventRecord(ws->gev_in, st));
        GX_CUDA(cudaStreamWaitEvent(gs, ws->gev_in, 0));
    }
    GX_CUDA(cudaGraphLaunch(g->exec, gs));
    count_launch(g->kernels);
    if (st != gs) {
        GX_CUDA(cudaEventRecord(ws->gev_out, gs));
        GX_CUDA(cudaStreamWaitEvent(st, ws->gev_out, 0));
    }
    return GX_SUCCESS;
}

}  // namespace

namespace gx {
gx_status search_launch(gx_index *ix, gx_workspace *ws, const gx_queries *q_dev, const gx_params *p, gx_result *out,
                        gx_cell *heap, uint32_t *hist, void *stream)
{
    return launch_search(ix, ws, q_dev, p, out, heap, hist, (cudaStream_t)stream);
}
void *workspace_stream(gx_workspace *ws) { return ws->stream; }
int32_t *workspace_err(gx_workspace *ws) { return ws->err; }
}  // namespace gx

extern "C" gx_status gx_workspace_set_tail(gx_workspace *ws, gx_tail_model *m, uint32_t sparse_below)
{
    if (!ws) return fail(GX_ERR_INVLD_PTR, "gx_workspace_set_tail: null workspace");
    ws->tail = m;
    ws->tail_below = m ? sparse_below : 0u;
    return GX_SUCCESS;
}

// ---- launch shape and its autotuner -------------------------------------------------------
namespace {

gx_tiles to_c(const BatchedTiles &t)
{
    return gx_tiles{(uint32_t)t.chunks, (uint32_t)t.ctas_per_sm, (uint32_t)t.tile, (uint32_t)t.sorted,
                    (uint32_t)t.pipeline};
}

BatchedTiles from_c(const gx_tiles &t)
{
    BatchedTiles b;
    b.chunks = (int)t.chunks_per_lane;
    b.ctas_per_sm = (int)t.ctas_per_sm;
    b.tile = (int)t.tile;
    b.sorted = (int)t.sorted;
    b.pipeline = (int)t.pipeline;
    return b;
}

// Workload shape the autotuner's choice is cached for: the index, and the parameters that
// decide the candidate windows and the scoring work of a spectrum.
struct TuneKey {
    const gx_index *ix;
    uint64_t dM_bits;   // the batch's tolerance (Da) bits; ~0 with per-spectrum tolerances
    uint32_t dF, min_shp, cap, flags, maxz;
    bool operator<(const TuneKey &o) const
    {
        return std::tie(ix, dM_bits, dF, min_shp, cap, flags, maxz) <
               std::tie(o.ix, o.dM_bits, o.dF, o.min_shp, o.cap, o.flags, o.maxz);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, BatchedTiles> g_tune_cache;

}  // namespace

extern "C" gx_status gx_workspace_set_graph(gx_workspace *ws, int32_t on)
{
    if (!ws) return fail(GX_ERR_INVLD_PTR, "gx_workspace_set_graph: null workspace");
    DeviceScope ds(ws->device);
    GX_CUDA(ds.status());
    if (on && !ws->gev_in) {
        GX_CUDA(cudaEventCreateWithFlags(&ws->gev_in, cudaEventDisableTiming));
        GX_CUDA(cudaEventCreateWithFlags(&ws->gev_out, cudaEventDisableTiming));
    }
    if (!on) {
        for (auto &g : ws->graphs) cudaGraphExecDestroy(g.exec);
        ws->graphs.clear();
    }
    ws->graph_on = on != 0;
    return GX_SUCCESS;
}

extern "C" gx_status gx_workspace_get_tiles(const gx_workspace *ws, gx_tiles *t)
{
    if (!ws || !t) return fail(GX_ERR_INVLD_PTR, "gx_workspace_get_tiles: null argument");
    *t = to_c(ws->tiles);
    return GX_SUCCESS;
}

extern "C" gx_status gx_workspace_set_tiles(gx_workspace *ws, const gx_tiles *t)
{
    if (!ws || !t) return fail(GX_ERR_INVLD_PTR, "gx_workspace_set_tiles: null argument");
    const BatchedTiles b = from_c(*t);
    if (!batched_tiles_valid(b, ws->tile) || (b.pipeline && !ws->bs.piped_ok[b.chunks]))
        return fail(GX_ERR_INVLD_PARAM, "gx_workspace_set_tiles: chunks_per_lane 1..3, ctas_per_sm 1..2, tile a "
                                        "multiple of 32 in 1024.." + std::to_string(ws->tile) + ", sorted 0 or 1, "
                                        "pipeline 0 or 1 (1 only with the whole block as the tile, where it fits)");
    ws->tiles = b;
    return GX_SUCCESS;
}

extern "C" gx_status gx_autotune(gx_index *ix, gx_workspace *ws, const gx_queries *q, const gx_params *p, uint32_t reps,
                                 uint32_t use_cache, gx_tune_result *out, void *stream)
{
    if (!ix || !ws || !q || !p || !out) return fail(GX_ERR_INVLD_PTR, "gx_autotune: null argument");
    if (ws->ix != ix) return fail(GX_ERR_INVLD_PARAM, "gx_autotune: workspace belongs to another index");
    if (p->flags & GX_FLAG_PLAIN) return fail(GX_ERR_INVLD_PARAM, "gx_autotune: the plain path has no tiles to tune");
    if (q->nspec == 0) return fail(GX_ERR_INVLD_SIZE, "gx_autotune: an empty sample");
    int32_t cap;
    gx_status rc = check_params(ix, p, &cap);
    if (rc != GX_SUCCESS) return rc;
    std::memset(out, 0, sizeof(*out));
    TuneKey key{ix, 0, p->dF, p->min_shp, (uint32_t)cap, p->flags, ix->maxz};
    if (q->dM) key.dM_bits = ~0ull;
    else std::memcpy(&key.dM_bits, &p->dM, sizeof(double));
    if (use_cache) {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end() && batched_tiles_valid(it->second, ws->tile)) {
            ws->tiles = it->second;
            out->best = to_c(it->second);
            out->cached = 1;
            return GX_SUCCESS;
        }
    }
    DeviceScope ds(ix->device);
    GX_CUDA(ds.status());
    cudaStream_t st = (cudaStream_t)stream;
    if (reps == 0) reps = 1;
    // candidates: id chunks per lane x CTAs per SM x tile width x spectrum order
    std::vector<BatchedTiles> cand;
    const int tiles[2] = {ws->tile, (ws->tile * 3 / 4) & ~31};
    for (int c = 1; c <= 3; c++)
        for (int k = 1; k <= 2; k++)
            for (int ti = 0; ti < 2; ti++)
                for (int so = 1; so >= 0; so--) {
                    BatchedTiles b;
                    b.chunks = c;
                    b.ctas_per_sm = k;
                    b.tile = tiles[ti];
                    b.sorted = so;
                    if (k <= ws->bs.max_ctas[c] && batched_tiles_valid(b, ws->tile) && cand.size() < GX_TUNE_MAX)
                        cand.push_back(b);
                }
    // the pipelined kernel (whole blocks as tiles; the batched kernel's share at two CTAs per SM)
    for (int c = 1; c <= 3; c++)
        for (int so = 1; so >= 0; so--) {
            BatchedTiles b;
            b.chunks = c;
            b.ctas_per_sm = 2;
            b.tile = ws->tile;
            b.sorted = so;
            b.pipeline = 1;
            if (ws->bs.piped_ok[c] && batched_tiles_valid(b, ws->tile) && cand.size() < GX_TUNE_MAX)
                cand.push_back(b);
        }
    const BatchedTiles keep = ws->tiles;
    std::vector<cudaEvent_t> ev(reps + 1);
    for (auto &e : ev) GX_CUDA(cudaEventCreate(&e));
    auto cleanup = [&]() {
        for (auto &e : ev) cudaEventDestroy(e);
    };
    float best_ms = INFINITY;
    BatchedTiles best = keep;
    for (size_t i = 0; i < cand.size(); i++) {
        ws->tiles = cand[i];
        rc = launch_search(ix, ws, q, p, ws->out, nullptr, nullptr, st);   // warm-up
        std::vector<float> t(reps);
        for (uint32_t r = 0; r < reps && rc == GX_SUCCESS; r++) {
            cudaEventRecord(ev[r], st);
            rc = launch_search(ix, ws, q, p, ws->out, nullptr, nullptr, st);
            cudaEventRecord(ev[r + 1], st);
        }
        cudaError_t e = cudaStreamSynchronize(st);
        if (rc != GX_SUCCESS || e != cudaSuccess) {
            ws->tiles = keep;
            cleanup();
            return rc != GX_SUCCESS ? rc : cuda_fail(e, "gx_autotune");
        }
        // back-to-back launches: each one's time is the gap between its two events
        for (uint32_t r = 0; r < reps; r++) cudaEventElapsedTime(&t[r], ev[r], ev[r + 1]);
        std::sort(t.begin(), t.end());
        const float ms = t[reps / 2];
        out->cand[i] = to_c(cand[i]);
        out->ms[i] = ms;
        if (ms < best_ms) {
            best_ms = ms;
            best = cand[i];
        }
    }
    cleanup();
    out->ncand = (uint32_t)cand.size();
    out->best = to_c(best);
    ws->tiles = best;
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        g_tune_cache[key] = best;
    }
    cudaGetLastError();
    return GX_SUCCESS;
}

extern "C" gx_status gx_search_device(gx_index *ix, gx_workspace *ws, const gx_queries *q, const gx_params *p,
                                      gx_result *out, gx_cell *heap, uint32_t *hist, void *stream)
{
    if (!ix || !ws || !q || !p || !out) return fail(GX_ERR_INVLD_PTR, "gx_search_device: null argument");
    if (ws->ix != ix) return fail(GX_ERR_INVLD_PARAM, "gx_search_device: workspace belongs to another index");
    DeviceScope ds(ix->device);
    GX_CUDA(ds.status());
    return launch_search(ix, ws, q, p, out, heap, hist, (cudaStream_t)stream);
}

extern "C" gx_status gx_search_host(gx_index *ix, gx_workspace *ws, const gx_queries *q, const gx_params *p,
                                    gx_result *out, gx_cell *heap_out, uint32_t *hist_out)
{
    if (!ix || !ws || !q || !p || !out) return fail(GX_ERR_INVLD_PTR, "gx_search_host: null argument");
    if (ws->ix != ix) return fail(GX_ERR_INVLD_PARAM, "gx_search_host: workspace belongs to another index");
    if (q->nspec > ws->max_spec || q->npeaks > ws->max_peaks)
        return fail(GX_ERR_INVLD_SIZE, "gx_search_host: batch larger than the workspace");
    if (q->nspec == 0) return GX_SUCCESS;
    if (!q->idx || !q->moz || !q->intn || !q->prec) return fail(GX_ERR_INVLD_PTR, "gx_search_host: null query array");
    if (q->idx[q->nspec] != q->npeaks) return fail(GX_ERR_INVLD_PARAM, "gx_search_host: idx[nspec] != npeaks");
    int32_t cap;
    gx_status rc = check_params(ix, p, &cap);
    if (rc != GX_SUCCESS) return rc;
    DeviceScope ds(ix->device);
    GX_CUDA(ds.status());
    cudaStream_t st = ws->stream;
    const uint32_t n = q->nspec;
    // the guard word may hold a flag of an earlier gx_search_device call, which reports none
    GX_CUDA(cudaMemsetAsync(ws->err, 0, sizeof(int32_t), st));
    if (heap_out && !ws->heap) GX_CUDA(cudaMalloc(&ws->heap, sizeof(gx_cell) * GX_MAX_HEAP * (uint64_t)ws->max_spec));
    if (hist_out && !ws->hist) GX_CUDA(cudaMalloc(&ws->hist, sizeof(uint32_t) * GX_HIST_BINS * (uint64_t)ws->max_spec));
    GX_CUDA(cudaMemcpyAsync(ws->qidx, q->idx, sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice, st));
    GX_CUDA(cudaMemcpyAsync(ws->moz, q->moz, sizeof(int32_t) * q->npeaks, cudaMemcpyHostToDevice, st));
    GX_CUDA(cudaMemcpyAsync(ws->intn, q->intn, sizeof(int32_t) * q->npeaks, cudaMemcpyHostToDevice, st));
    GX_CUDA(cudaMemcpyAsync(ws->prec, q->prec, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    if (q->dM) GX_CUDA(cudaMemcpyAsync(ws->dMq, q->dM, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    gx_queries dq = *q;
    dq.idx = ws->qidx; dq.moz = ws->moz; dq.intn = ws->intn; dq.prec = ws->prec;
    if (q->charge) GX_CUDA(cudaMemcpyAsync(ws->charge, q->charge, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
    dq.charge = q->charge ? ws->charge : nullptr;
    dq.dM = q->dM ? ws->dMq : nullptr;
    rc = launch_search(ix, ws, &dq, p, ws->out, heap_out ? ws->heap : nullptr, hist_out ? ws->hist : nullptr, st);
    if (rc != GX_SUCCESS) return rc;
    GX_CUDA(cudaMemcpyAsync(out, ws->out, sizeof(gx_result) * n, cudaMemcpyDeviceToHost, st));
    if (heap_out)
        GX_CUDA(cudaMemcpyAsync(heap_out, ws->heap, sizeof(gx_cell) * cap * (uint64_t)n, cudaMemcpyDeviceToHost, st));
    if (hist_out)
        GX_CUDA(cudaMemcpyAsync(hist_out, ws->hist, sizeof(uint32_t) * GX_HIST_BINS * (uint64_t)n,
                                cudaMemcpyDeviceToHost, st));
    int32_t err = 0;
    GX_CUDA(cudaMemcpyAsync(&err, ws->err, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GX_CUDA(cudaStreamSynchronize(st));
    if (err) {
        cudaMemsetAsync(ws->err, 0, sizeof(int32_t), st);
        return fail(GX_ERR_DEVICE_GUARD, "a spectrum has more peaks than GX_MAX_PEAKS");
    }
    return GX_SUCCESS;
}
