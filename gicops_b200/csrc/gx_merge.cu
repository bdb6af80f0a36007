// Merge step of an index-sharded search on the GPU.  Each rank holds a subset of the
// peptide lengths and searches every spectrum against it (the reference's distributed
// design, where MPI ranks own peptide subsets and exchange partial results through
// files: source/core/lbe_internal.cpp:75-103, source/core/dslim_score.cpp:199-388).
// After the collectives (the per-spectrum histograms and candidate counts summed, every
// rank's top-k cells and statuses gathered), one warp per spectrum:
//   - selects the global top `cap` cells from world*k, ordered by hyperscore descending,
//     then global length index and entry ascending, mapping each rank's local length
//     index to the global one;
//   - writes the result record as a single-index search would: candidate count, the
//     status bits of the ranks' scorecards, the top cell, and the tail fit and e-value
//     of the summed histogram (the fit depends only on the histogram, the count and the
//     top hyperscore, which equal the single-index ones).
// With ties in the top hyperscore the reported top cell may differ from the one a
// single heap's getMax picks; its hyperscore, and so the e-value, do not.

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "../../include/gicops_b200.h"
#include "gx_device.cuh"
#include "gx_internal.h"

namespace gx {

constexpr int kMergeWarps = 4;

struct MKey {          // order: hyperscore descending, then global length, then entry
    uint32_t hi;       // ~float bits of a positive hyperscore (ascending = h descending)
    uint32_t ixx;
    int32_t psid;
};

__device__ __forceinline__ bool key_less(const MKey &a, const MKey &b)
{
    if (a.hi != b.hi) return a.hi < b.hi;
    if (a.ixx != b.ixx) return a.ixx < b.ixx;
    return a.psid < b.psid;
}

__global__ void __launch_bounds__(kMergeWarps * 32)
    k_merge_shards(uint32_t n, int world, int k, int cap, const gx_cell *__restrict__ cells,
                   const int32_t *__restrict__ status, const uint16_t *__restrict__ lut,
                   const uint32_t *__restrict__ hist, const int32_t *__restrict__ cpsms, uint32_t min_cpsm,
                   double expect_max, gx_cell *top, gx_result *out)
{
    __shared__ uint32_t h[kMergeWarps][kHist];
    __shared__ double sx[kMergeWarps][kHist + 2];
    __shared__ gx_cell best[kMergeWarps][GX_MAX_HEAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t s = blockIdx.x * kMergeWarps + w;
    if (s >= n) return;
    const int total = world * k;
    // ---- selection: cap rounds of a warp-wide minimum above the last key taken -------
    MKey prev{0u, 0u, -1};
    bool any_prev = false;
    int taken = 0;
    for (; taken < cap; taken++) {
        MKey bk{0xFFFFFFFFu, 0xFFFFFFFFu, 0x7FFFFFFF};
        int bi = -1;
        for (int c = lane; c < total; c += 32) {
            const int r = c / k, j = c - r * k;
            const gx_cell x = cells[((uint64_t)r * n + s) * k + j];
            if (!(x.hyperscore > 0.0f) || x.idxoffset >= GX_MAX_LENGTHS) continue;   // empty cell
            const MKey kk{~__float_as_uint(x.hyperscore), (uint32_t)lut[r * GX_MAX_LENGTHS + x.idxoffset], x.psid};
            if (any_prev && !key_less(prev, kk)) continue;
            if (bi < 0 || key_less(kk, bk)) {
                bk = kk;
                bi = c;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            MKey ok;
            ok.hi = __shfl_xor_sync(0xffffffffu, bk.hi, o);
            ok.ixx = __shfl_xor_sync(0xffffffffu, bk.ixx, o);
            ok.psid = __shfl_xor_sync(0xffffffffu, bk.psid, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (oi >= 0 && (bi < 0 || key_less(ok, bk))) {
                bk = ok;
                bi = oi;
            }
        }
        if (bi < 0) break;   // fewer than cap non-empty cells
        if (lane == 0) {
            const int r = bi / k, j = bi - r * k;
            gx_cell x = cells[((uint64_t)r * n + s) * k + j];
            x.idxoffset = (uint16_t)bk.ixx;
            best[w][taken] = x;
        }
        prev = bk;
        any_prev = true;
    }
    __syncwarp();
    if (top)
        for (int t = lane; t < cap; t += 32) top[(uint64_t)s * cap + t] = t < taken ? best[w][t] : gx_cell{};
    // ---- result record and tail fit of the summed histogram -------------------------
    gx_result r;
    memset(&r, 0, sizeof(r));
    r.cpsms = cpsms[s];
    int32_t st = 0;
    for (int q = 0; q < world; q++) st |= status[(uint64_t)q * n + s] & (4 | 8);
    r.status = st;
    if (fits_tail(r.cpsms, min_cpsm) && taken > 0) {
        r.top = best[w][0];
        r.maxhyp = __double2int_rz(__dadd_rn((double)__fmul_rn(r.top.hyperscore, 10.0f), 0.5));
        for (int b = lane; b < kHist; b += 32) h[w][b] = hist[(uint64_t)s * kHist + b];
        __syncwarp();
        tail_fit_warp(h[w], r.cpsms, r.maxhyp, sx[w], r, lane);
        r.status |= 1;
        if (r.e_x < expect_max) r.status |= 2;
    }
    if (lane == 0) out[s] = r;
}

}  // namespace gx

using namespace gx;

extern "C" gx_status gx_merge_shards_device(uint32_t nspec, int32_t world, uint32_t k, const gx_cell *cells_dev,
                                            const int32_t *status_dev, const uint16_t *lut_dev,
                                            const uint32_t *hist_dev, const int32_t *cpsms_dev, const gx_params *p,
                                            gx_cell *top_dev, gx_result *out_dev, void *stream)
{
    if (!p || (nspec && (!cells_dev || !status_dev || !lut_dev || !hist_dev || !cpsms_dev || !out_dev)))
        return fail(GX_ERR_INVLD_PTR, "gx_merge_shards_device: null argument");
    if (world < 1 || world > 1024 || k < 1 || k > (uint32_t)GX_MAX_HEAP)
        return fail(GX_ERR_INVLD_PARAM, "gx_merge_shards_device: world must be 1..1024 and k 1..GX_MAX_HEAP");
    const int32_t cap = gx_heap_capacity(p->topmatches);
    if (cap < 1 || cap > GX_MAX_HEAP)
        return fail(GX_ERR_INVLD_PARAM, "gx_merge_shards_device: topmatches gives no usable heap capacity");
    if (nspec == 0) return GX_SUCCESS;
    cudaGetLastError();   // an earlier call's error is not ours to report
    k_merge_shards<<<(nspec + kMergeWarps - 1) / kMergeWarps, kMergeWarps * 32, 0, (cudaStream_t)stream>>>(
        nspec, world, (int)k, cap, cells_dev, status_dev, lut_dev, hist_dev, cpsms_dev, p->min_cpsm, p->expect_max,
        top_dev, out_dev);
    count_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GX_SUCCESS : cuda_fail(e, "gx_merge_shards_device");
}
