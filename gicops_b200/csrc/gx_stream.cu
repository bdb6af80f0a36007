// Streamed search of a batch held in host memory, in chunks, with the copies of one
// chunk overlapping the search of another.
//
// The reference feeds its GPU path one batch at a time from a ring of host query buffers
// (source/core/dslim_query.cpp:183-203), uploading each batch synchronously before its
// search (dQueries::H2D, source/core/cuda/superstep3/kernel.cu:192-206).  Here a host
// batch of any size is cut into chunks of at most `chunk` spectra that cycle through two
// sets of device buffers:
//
//   upload stream    H2D of chunk i's arrays (one cudaMemcpyAsync per array) into set i%2,
//                    once the search of chunk i-2 (the set's previous user) is done
//   search stream    rebase chunk i's peak offsets to 0, search (the workspace's launch
//                    sequence: k_prep, sort, k_search_batched, k_tailfit, learned tail),
//                    once its upload and the download of chunk i-2's results are done
//   download stream  D2H of chunk i's results into the caller's array
//
// Every per-spectrum result is independent of the batch it was searched in, so the
// results equal those of one search over the whole batch.

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/gicops_b200.h"
#include "gx_device_scope.cuh"
#include "gx_index.cuh"
#include "gx_internal.h"

namespace gx {
namespace {

// idx[i] -= base for the n + 1 offsets of a chunk (its peaks are copied from `base` on)
__global__ void k_rebase(uint32_t *idx, uint32_t n1, uint32_t base)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n1) idx[i] -= base;
}

struct Buffers {
    uint32_t *idx = nullptr;
    int32_t *moz = nullptr, *intn = nullptr, *charge = nullptr;
    float *prec = nullptr;
    double *dM = nullptr;
    gx_result *out = nullptr;
};

}  // namespace
}  // namespace gx

using namespace gx;

struct gx_streamer {
    gx_index *ix = nullptr;
    gx_workspace *ws = nullptr;
    int device = 0;
    uint32_t chunk = 0, max_peaks = 0;
    Buffers buf[2];
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t uploaded[2] = {}, searched[2] = {}, downloaded[2] = {};
    std::vector<void *> allocs;
};

extern "C" gx_status gx_streamer_free(gx_streamer *s)
{
    if (!s) return GX_SUCCESS;
    DeviceScope ds(s->device);
    if (s->up) cudaStreamSynchronize(s->up);
    if (s->down) cudaStreamSynchronize(s->down);
    for (void *p : s->allocs) cudaFree(p);
    for (int b = 0; b < 2; b++) {
        if (s->uploaded[b]) cudaEventDestroy(s->uploaded[b]);
        if (s->searched[b]) cudaEventDestroy(s->searched[b]);
        if (s->downloaded[b]) cudaEventDestroy(s->downloaded[b]);
    }
    if (s->up) cudaStreamDestroy(s->up);
    if (s->down) cudaStreamDestroy(s->down);
    gx_workspace_free(s->ws);
    delete s;
    cudaGetLastError();   // nothing of a free is reported to the next call
    return GX_SUCCESS;
}

extern "C" gx_status gx_streamer_create(gx_index *ix, uint32_t chunk, uint32_t max_peaks, gx_streamer **out)
{
    if (!ix || !out) return fail(GX_ERR_INVLD_PTR, "gx_streamer_create: null argument");
    *out = nullptr;
    if (chunk == 0) return fail(GX_ERR_INVLD_PARAM, "gx_streamer_create: chunk must be > 0");
    if (max_peaks == 0) max_peaks = chunk * 160u;
    DeviceScope ds(ix->device);
    if (ds.status() != cudaSuccess) return cuda_fail(ds.status(), "gx_streamer_create: cudaSetDevice");
    cudaGetLastError();
    auto *s = new gx_streamer();
    s->ix = ix;
    s->device = ix->device;
    s->chunk = chunk;
    s->max_peaks = max_peaks;
    gx_status st = gx_workspace_create(ix, chunk, max_peaks, &s->ws);
    if (st != GX_SUCCESS) {
        delete s;
        return st;
    }
    cudaError_t e = cudaSuccess;
    auto al = [&](auto **p, size_t count) {
        void *q = nullptr;
        if (e == cudaSuccess) e = cudaMalloc(&q, count * sizeof(**p) + 16);
        if (e == cudaSuccess) s->allocs.push_back(q);
        *p = static_cast<std::remove_reference_t<decltype(*p)>>(q);
    };
    for (auto &b : s->buf) {
        al(&b.idx, (size_t)chunk + 1);
        al(&b.moz, max_peaks);
        al(&b.intn, max_peaks);
        al(&b.charge, chunk);
        al(&b.prec, chunk);
        al(&b.dM, chunk);
        al(&b.out, chunk);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->up, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->down, cudaStreamNonBlocking);
    for (int b = 0; b < 2 && e == cudaSuccess; b++) {
        e = cudaEventCreateWithFlags(&s->uploaded[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->searched[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->downloaded[b], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        gx_streamer_free(s);
        return fail(GX_ERR_BAD_MEM_ALLOC, std::string("gx_streamer_create: ") + cudaGetErrorString(e));
    }
    *out = s;
    return GX_SUCCESS;
}

extern "C" gx_workspace *gx_streamer_workspace(gx_streamer *s) { return s ? s->ws : nullptr; }

extern "C" gx_status gx_search_stream(gx_streamer *s, const gx_queries *q, const gx_params *p, gx_result *out,
                                      gx_stream_stats *stats)
{
    if (!s || !q || !p || !out) return fail(GX_ERR_INVLD_PTR, "gx_search_stream: null argument");
    if (stats) *stats = gx_stream_stats{};
    if (q->nspec == 0) return GX_SUCCESS;
    if (!q->idx || !q->moz || !q->intn || !q->prec) return fail(GX_ERR_INVLD_PTR, "gx_search_stream: null query array");
    if (q->idx[0] != 0 || q->idx[q->nspec] != q->npeaks)
        return fail(GX_ERR_INVLD_PARAM, "gx_search_stream: idx[0] must be 0 and idx[nspec] == npeaks");
    const uint32_t nchunks = (q->nspec + s->chunk - 1) / s->chunk;
    for (uint32_t c = 0; c < nchunks; c++) {   // every chunk must fit its buffers before any work
        const uint32_t c0 = c * s->chunk, c1 = c0 + s->chunk < q->nspec ? c0 + s->chunk : q->nspec;
        if (q->idx[c1] < q->idx[c0]) return fail(GX_ERR_INVLD_PARAM, "gx_search_stream: idx must not decrease");
        if (q->idx[c1] - q->idx[c0] > s->max_peaks)
            return fail(GX_ERR_INVLD_SIZE, "gx_search_stream: chunk " + std::to_string(c) + " has " +
                                               std::to_string(q->idx[c1] - q->idx[c0]) +
                                               " peaks, more than the streamer's " + std::to_string(s->max_peaks));
    }
    DeviceScope ds(s->device);
    if (ds.status() != cudaSuccess) return cuda_fail(ds.status(), "gx_search_stream: cudaSetDevice");
    cudaGetLastError();   // an earlier call's error is not ours to report
    cudaStream_t ks = (cudaStream_t)workspace_stream(s->ws);
    int32_t *err = workspace_err(s->ws);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int32_t), ks);
    // timing (optional): events bracketing each chunk's upload, search and download
    std::vector<cudaEvent_t> tev;
    auto mark = [&](cudaStream_t st) -> int {
        if (!stats || e != cudaSuccess) return -1;
        cudaEvent_t ev;
        if ((e = cudaEventCreate(&ev)) != cudaSuccess) return -1;
        tev.push_back(ev);
        e = cudaEventRecord(ev, st);
        return (int)tev.size() - 1;
    };
    struct Span { int a, b; };
    std::vector<Span> sp_up, sp_search, sp_down;
    const int t_start = mark(s->up);
    gx_status rc = GX_SUCCESS;
    for (uint32_t c = 0; c < nchunks && e == cudaSuccess && rc == GX_SUCCESS; c++) {
        const int b = (int)(c & 1u);
        Buffers &B = s->buf[b];
        const uint32_t c0 = c * s->chunk, c1 = c0 + s->chunk < q->nspec ? c0 + s->chunk : q->nspec, n = c1 - c0;
        const uint32_t p0 = q->idx[c0], np = q->idx[c1] - p0;
        // upload: the set's previous chunk (c - 2) must be searched
        if (c >= 2) e = cudaStreamWaitEvent(s->up, s->searched[b], 0);
        const int u0 = mark(s->up);
        auto h2d = [&](void *dst, const void *src, size_t bytes) {
            if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s->up);
        };
        h2d(B.idx, q->idx + c0, sizeof(uint32_t) * ((size_t)n + 1));
        h2d(B.moz, q->moz + p0, sizeof(int32_t) * (size_t)np);
        h2d(B.intn, q->intn + p0, sizeof(int32_t) * (size_t)np);
        h2d(B.prec, q->prec + c0, sizeof(float) * (size_t)n);
        if (q->charge) h2d(B.charge, q->charge + c0, sizeof(int32_t) * (size_t)n);
        if (q->dM) h2d(B.dM, q->dM + c0, sizeof(double) * (size_t)n);
        const int u1 = mark(s->up);
        if (e == cudaSuccess) e = cudaEventRecord(s->uploaded[b], s->up);
        // search: after the upload, and after the set's results of chunk c - 2 are downloaded
        if (e == cudaSuccess) e = cudaStreamWaitEvent(ks, s->uploaded[b], 0);
        if (e == cudaSuccess && c >= 2) e = cudaStreamWaitEvent(ks, s->downloaded[b], 0);
        if (e != cudaSuccess) break;
        const int k0 = mark(ks);
        k_rebase<<<(n + 1 + 255) / 256, 256, 0, ks>>>(B.idx, n + 1, p0);
        count_launch();
        gx_queries dq{};
        dq.nspec = n;
        dq.npeaks = np;
        dq.idx = B.idx;
        dq.moz = B.moz;
        dq.intn = B.intn;
        dq.prec = B.prec;
        dq.charge = q->charge ? B.charge : nullptr;
        dq.dM = q->dM ? B.dM : nullptr;
        rc = search_launch(s->ix, s->ws, &dq, p, B.out, nullptr, nullptr, ks);
        if (rc != GX_SUCCESS) break;
        const int k1 = mark(ks);
        if (e == cudaSuccess) e = cudaEventRecord(s->searched[b], ks);
        // download
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s->down, s->searched[b], 0);
        const int d0 = mark(s->down);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(out + c0, B.out, sizeof(gx_result) * (size_t)n, cudaMemcpyDeviceToHost, s->down);
        const int d1 = mark(s->down);
        if (e == cudaSuccess) e = cudaEventRecord(s->downloaded[b], s->down);
        if (stats) {
            sp_up.push_back({u0, u1});
            sp_search.push_back({k0, k1});
            sp_down.push_back({d0, d1});
        }
    }
    const int t_end = mark(s->down);
    int32_t guard = 0;
    cudaError_t e2 = cudaStreamSynchronize(s->up);
    if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(ks);
    if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(s->down);
    if (e2 == cudaSuccess) e2 = cudaMemcpy(&guard, err, sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (stats && e == cudaSuccess && e2 == cudaSuccess && rc == GX_SUCCESS) {
        auto ms = [&](int a, int b) {
            float v = 0.0f;
            if (a >= 0 && b >= 0) cudaEventElapsedTime(&v, tev[a], tev[b]);
            return (double)v;
        };
        stats->chunks = nchunks;
        stats->total_ms = ms(t_start, t_end);
        for (size_t i = 0; i < sp_up.size(); i++) {
            stats->upload_ms += ms(sp_up[i].a, sp_up[i].b);
            stats->search_ms += ms(sp_search[i].a, sp_search[i].b);
            stats->download_ms += ms(sp_down[i].a, sp_down[i].b);
        }
    }
    for (cudaEvent_t ev : tev) cudaEventDestroy(ev);
    if (rc != GX_SUCCESS) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "gx_search_stream");
    if (e2 != cudaSuccess) return cuda_fail(e2, "gx_search_stream: synchronise");
    if (guard) {
        cudaMemset(err, 0, sizeof(int32_t));
        return fail(GX_ERR_DEVICE_GUARD, "gx_search_stream: a spectrum has more peaks than GX_MAX_PEAKS");
    }
    return GX_SUCCESS;
}
