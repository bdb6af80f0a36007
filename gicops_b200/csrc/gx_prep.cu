// Query preprocessing on the GPU: peak picking and intensity normalisation of raw
// spectra (the reference's MSQuery::pickpeaks, source/core/msquery.cpp:338-423, as its
// MS2 -> .pbin conversion runs it), one thread per spectrum, then the kept peaks
// gathered into the CSR query batch the search reads.
//
// The reference sorts each spectrum's (intensity, m/z) pairs with its own key-value
// quicksort (source/core/include/keyval.h:49-129: Hoare partition around the middle
// element, both sides recursed).  Equal intensities end in the order that partition
// sequence leaves them, which decides which tied peaks survive the 100-peak cut and the
// order they are written in, so the same partition steps are run here.  The ranges a
// partition leaves are disjoint, so the order they are sorted in does not matter: the
// smaller is sorted first and the larger kept on a stack, which stays within
// log2(size) + 1 entries.

#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/gicops_b200.h"
#include "gx_internal.h"

namespace gx {

// double -> int32 as x86's truncating conversion does it (the reference's implicit
// int casts): out of range and NaN give INT32_MIN.
__device__ __forceinline__ int32_t cvt_i32(double v)
{
    return (v >= -2147483648.0 && v < 2147483648.0) ? (int32_t)v : INT32_MIN;
}

constexpr int kSortStack = 40;   // > log2(2^31) + 1: the stack never fills

__device__ void kv_sort(int32_t *key, int32_t *val, int n)
{
    int st_l[kSortStack], st_r[kSortStack];
    int sp = 0;
    int left = 0, right = n - 1;
    for (;;) {
        if (left < right) {
            int i = left, j = right;
            const int32_t pivot = key[left + (right - left) / 2];
            while (i <= j) {
                while (key[i] < pivot) i++;
                while (key[j] > pivot) j--;
                if (i <= j) {
                    const int32_t tk = key[i], tv = val[i];
                    key[i] = key[j];
                    val[i] = val[j];
                    key[j] = tk;
                    val[j] = tv;
                    i++;
                    j--;
                }
            }
            // sides [left, j] and [i, right]: sort the smaller now, stack the larger
            const bool a = left < j, b = i < right;
            if (a && b && sp < kSortStack) {
                if (j - left < right - i) {
                    st_l[sp] = i; st_r[sp] = right; sp++;
                    right = j;
                } else {
                    st_l[sp] = left; st_r[sp] = j; sp++;
                    left = i;
                }
                continue;
            }
            if (a) { right = j; continue; }
            if (b) { left = i; continue; }
        }
        if (sp == 0) return;
        sp--;
        left = st_l[sp];
        right = st_r[sp];
    }
}

// One thread per spectrum: sort, scale, count the kept peaks into kept[s] (= out_idx[s + 1]).
__global__ void k_pick(uint32_t nspec, const uint32_t *__restrict__ seg, const uint32_t *__restrict__ size,
                       int32_t *mz, int32_t *intn, int32_t base_int, int32_t min_int, int qalen, uint32_t *kept)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nspec) return;
    const uint32_t a = seg[s], b = seg[s + 1];
    const uint32_t nvec = b > a ? b - a : 0u;
    const int S = (int)min(size[s], nvec);   // a size beyond the segment is clamped
    int k = 0;
    if (S > 0) {
        int32_t *in = intn + a, *m = mz + a;
        kv_sort(in, m, S);
        const double factor = (double)base_int / (double)in[S - 1];
        in[S - 1] = base_int;
        k = 1;
        for (int j = S - 2; j >= S - qalen && j >= 0; j--) {
            in[j] = cvt_i32((double)in[j] * factor);
            if (in[j] >= min_int)
                k++;
            else
                break;
        }
        if (k >= qalen) k = qalen;
    }
    kept[s] = (uint32_t)k;
    if (s == 0) kept[-1] = 0u;   // out_idx[0]
}

// One warp per spectrum: the last kept values of its segment, in order.
__global__ void k_gather_kept(uint32_t nspec, const uint32_t *__restrict__ seg, const uint32_t *__restrict__ out_idx,
                              const int32_t *__restrict__ mz, const int32_t *__restrict__ intn, int32_t *out_mz,
                              int32_t *out_intn)
{
    const uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= nspec) return;
    const uint32_t o = out_idx[s], k = out_idx[s + 1] - o, b = seg[s + 1];
    for (uint32_t i = lane; i < k; i += 32) {
        out_mz[o + i] = mz[b - k + i];
        out_intn[o + i] = intn[b - k + i];
    }
}

}  // namespace gx

using namespace gx;

extern "C" gx_status gx_pickpeaks_device(uint32_t nspec, const uint32_t *seg_dev, const uint32_t *size_dev,
                                         int32_t *mz_dev, int32_t *intn_dev, int32_t base_int, int32_t min_int,
                                         uint32_t qalen, uint32_t *out_idx_dev, int32_t *out_mz_dev,
                                         int32_t *out_intn_dev, void *stream)
{
    if (!out_idx_dev) return fail(GX_ERR_INVLD_PTR, "gx_pickpeaks_device: null out_idx");
    if (nspec && (!seg_dev || !size_dev || !mz_dev || !intn_dev || !out_mz_dev || !out_intn_dev))
        return fail(GX_ERR_INVLD_PTR, "gx_pickpeaks_device: null argument");
    if (qalen < 1 || qalen > (1u << 30)) return fail(GX_ERR_INVLD_PARAM, "gx_pickpeaks_device: qalen must be >= 1");
    if (nspec >= (1u << 31)) return fail(GX_ERR_INVLD_SIZE, "gx_pickpeaks_device: 2^31 or more spectra");
    cudaGetLastError();   // an earlier call's error is not ours to report
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    if (nspec == 0) {
        e = cudaMemsetAsync(out_idx_dev, 0, sizeof(uint32_t), st);
        return e == cudaSuccess ? GX_SUCCESS : cuda_fail(e, "gx_pickpeaks_device");
    }
    size_t tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, out_idx_dev + 1, out_idx_dev + 1, (int)nspec);
    void *tmp = nullptr;
    if ((e = cudaMallocAsync(&tmp, tb ? tb : 16, st)) != cudaSuccess) {
        cudaGetLastError();
        return fail(GX_ERR_BAD_MEM_ALLOC, "gx_pickpeaks_device: scan scratch");
    }
    k_pick<<<(nspec + 127) / 128, 128, 0, st>>>(nspec, seg_dev, size_dev, mz_dev, intn_dev, base_int, min_int,
                                                (int)qalen, out_idx_dev + 1);
    count_launch();
    e = cub::DeviceScan::InclusiveSum(tmp, tb, out_idx_dev + 1, out_idx_dev + 1, (int)nspec, st);
    count_launch();
    if (e == cudaSuccess) {
        const uint64_t threads = (uint64_t)nspec * 32;
        k_gather_kept<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(nspec, seg_dev, out_idx_dev, mz_dev, intn_dev,
                                                                          out_mz_dev, out_intn_dev);
        count_launch();
        e = cudaGetLastError();
    }
    cudaFreeAsync(tmp, st);
    if (e != cudaSuccess) return cuda_fail(e, "gx_pickpeaks_device");
    return GX_SUCCESS;
}
