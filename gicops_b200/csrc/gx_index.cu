// Index residency in HBM (the counterpart of the reference's s1::getdIndex,
// source/core/cuda/superstep1/kernel.cu:310-358): the per-length arrays are copied
// once, then two device-side forms are derived from them:
//
//   iA   the reference's bin-major CSR (bA offsets unchanged) with each ion id
//        entry*speclen + pos rewritten as 2*entry + (pos >= speclen/2): the entry and
//        its ion series, which is all the query path reads from an id.  Order inside
//        a bucket is unchanged (the plain path probes it with binary searches).
//   iAb  the same ids regrouped by blocks of `block` consecutive entries: inside each
//        block a CSR over the same bins (offsets blkA[block][bin], bins 0..nbins), each
//        id stored as 16 bits relative to its block, 2*(entry - block start) + (y ion).
//        A candidate tile of the batched path is one block, so every bin range of a
//        probed interval is one contiguous run of exactly the tile's ids, read as
//        16-byte chunks of 8 ids (the allocation is padded by one chunk).

#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gicops_b200.h"
#include "gx_device.cuh"
#include "gx_index.cuh"
#include "gx_internal.h"

namespace gx {

__global__ void k_encode_ids(uint32_t *iA, uint64_t n, uint32_t speclen, uint32_t half, uint32_t magic)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t id = iA[i];
        const uint32_t e = div_speclen(id, speclen, magic);
        iA[i] = 2u * e + ((id - e * speclen) >= half ? 1u : 0u);
    }
}

__device__ __forceinline__ uint32_t lb(const uint32_t *v, uint32_t a, uint32_t b, uint32_t key)
{
    while (a < b) {
        const uint32_t c = a + ((b - a) >> 1);
        if (v[c] < key) a = c + 1; else b = c;
    }
    return a;
}

// counts[k][b] = ids of bucket b whose entry lies in block k (rows of nbins + 1; the
// last column stays 0 so that an exclusive scan yields each block's end offset there).
__global__ void k_blk_count(const uint32_t *iA, const uint32_t *bA, uint32_t nbins, uint32_t E, uint32_t nblk,
                            uint32_t *counts)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > nbins) return;
    const uint64_t row = (uint64_t)nbins + 1;
    if (b + 1 >= nbins) {
        for (uint32_t k = 0; k < nblk; k++) counts[k * row + b] = 0;
        return;
    }
    const uint32_t s = bA[b], e = bA[b + 1];
    uint32_t prev = s;
    for (uint32_t k = 0; k < nblk; k++) {
        const uint64_t key64 = 2ull * (uint64_t)(k + 1) * E;
        const uint32_t p = key64 >= 0xFFFFFFFFull ? e : lb(iA, prev, e, (uint32_t)key64);
        counts[k * row + b] = p - prev;
        prev = p;
    }
}

__global__ void k_blk_scatter(const uint32_t *iA, const uint32_t *bA, const uint32_t *offs, uint32_t nbins, uint32_t E,
                              uint32_t nblk, uint16_t *iAb)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b + 1 >= nbins) return;
    const uint64_t row = (uint64_t)nbins + 1;
    const uint32_t s = bA[b], e = bA[b + 1];
    uint32_t prev = s;
    for (uint32_t k = 0; k < nblk; k++) {
        const uint64_t key64 = 2ull * (uint64_t)(k + 1) * E;
        const uint32_t p = key64 >= 0xFFFFFFFFull ? e : lb(iA, prev, e, (uint32_t)key64);
        uint32_t d = offs[k * row + b];
        const uint32_t lo = 2u * k * E;
        for (uint32_t i = prev; i < p; i++) iAb[d++] = (uint16_t)(iA[i] - lo);
        prev = p;
    }
}

}  // namespace gx

using namespace gx;

extern "C" gx_status gx_index_free(gx_index *ix)
{
    if (!ix) return GX_SUCCESS;
    cudaSetDevice(ix->device);
    cudaFree(ix->bA);
    cudaFree(ix->iA);
    cudaFree(ix->iAb);
    cudaFree(ix->blkA);
    cudaFree(ix->mass);
    cudaFree(ix->lens);
    delete ix;
    return GX_SUCCESS;
}

extern "C" uint64_t gx_index_bytes(const gx_index *ix) { return ix ? ix->bytes : 0; }

extern "C" gx_status gx_index_upload(const gx_length_desc *lens, int32_t nlen, uint32_t nbins, int32_t device,
                                     gx_index **out)
{
    if (!lens || !out) return fail(GX_ERR_INVLD_PTR, "gx_index_upload: null argument");
    *out = nullptr;
    if (nlen < 1 || nlen > GX_MAX_LENGTHS || nbins < 2)
        return fail(GX_ERR_INVLD_PARAM, "gx_index_upload: nlen must be 1..64 and nbins >= 2");
    const uint32_t E = (uint32_t)kBlockEntries;
    uint32_t maxz = 0;
    uint64_t tot_ia = 0, tot_m = 0, tot_blk = 0;
    std::vector<DevLen> hl(nlen);
    for (int i = 0; i < nlen; i++) {
        const gx_length_desc &d = lens[i];
        if (d.peplen < 2 || d.speclen < 2 || d.speclen % (2 * (d.peplen - 1)) != 0)
            return fail(GX_ERR_INVLD_INDEX, "gx_index_upload: speclen must be 2*(L-1)*maxz");
        const uint32_t z = d.speclen / (2 * (d.peplen - 1));
        if (maxz && z != maxz) return fail(GX_ERR_INVLD_INDEX, "gx_index_upload: lengths disagree on maxz");
        maxz = z;
        if ((uint64_t)d.npep * d.speclen >= (1ull << 32) - 16 || d.npep >= (1u << 31))
            return fail(GX_ERR_INVLD_SIZE, "gx_index_upload: 2^32 - 16 or more ion ids in one length");
        if (d.npep && (!d.mass || !d.bA || !d.iA)) return fail(GX_ERR_INVLD_PTR, "gx_index_upload: null array");
        if (!d.bA) return fail(GX_ERR_INVLD_PTR, "gx_index_upload: null bA");
        if (d.bA[nbins - 1] != (uint64_t)d.npep * d.speclen)
            return fail(GX_ERR_INVLD_INDEX, "gx_index_upload: bA[nbins-1] must equal npep*speclen");
        const uint32_t magic = (uint32_t)(((1ull << 32) + d.speclen - 1) / d.speclen);
        const uint32_t nblk = d.npep ? (d.npep + E - 1) / E : 0;
        hl[i] = DevLen{tot_ia, tot_m, d.npep, d.speclen, d.speclen / 2, d.peplen, magic, nblk, tot_blk};
        tot_ia += (uint64_t)d.npep * d.speclen;
        tot_m += d.npep;
        tot_blk += (uint64_t)nblk * (nbins + 1);
    }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "gx_index_upload: cudaSetDevice");
    auto *ix = new gx_index();
    ix->device = device;
    ix->nlen = nlen;
    ix->nbins = nbins;
    ix->maxz = maxz;
    ix->block = E;
    ix->hlens = hl;
    auto cleanup = [&](gx_status st) {
        gx_index_free(ix);
        return st;
    };
    if ((e = cudaMalloc(&ix->bA, sizeof(uint32_t) * (uint64_t)nbins * nlen)) != cudaSuccess ||
        (e = cudaMalloc(&ix->iA, sizeof(uint32_t) * (tot_ia ? tot_ia : 1))) != cudaSuccess ||
        (e = cudaMalloc(&ix->iAb, sizeof(uint16_t) * (tot_ia + 8))) != cudaSuccess ||
        (e = cudaMalloc(&ix->blkA, sizeof(uint32_t) * (tot_blk ? tot_blk : 1))) != cudaSuccess ||
        (e = cudaMalloc(&ix->mass, sizeof(float) * (tot_m ? tot_m : 1))) != cudaSuccess ||
        (e = cudaMalloc(&ix->lens, sizeof(DevLen) * nlen)) != cudaSuccess) {
        cudaGetLastError();
        return cleanup(fail(GX_ERR_BAD_MEM_ALLOC, std::string("gx_index_upload: ") + cudaGetErrorString(e)));
    }
    ix->bytes = sizeof(uint32_t) * ((uint64_t)nbins * nlen + tot_ia + tot_blk) + sizeof(uint16_t) * (tot_ia + 8) +
                sizeof(float) * tot_m + sizeof(DevLen) * nlen;
    ix->iab_bytes = sizeof(uint16_t) * tot_ia;
    if ((e = cudaMemset(ix->iAb + tot_ia, 0, 8 * sizeof(uint16_t))) != cudaSuccess)
        return cleanup(cuda_fail(e, "gx_index_upload: iAb padding"));
    // scan scratch, sized for the largest per-length offset table
    uint64_t max_rows = 1;
    for (int i = 0; i < nlen; i++) max_rows = std::max<uint64_t>(max_rows, (uint64_t)hl[i].nblk * (nbins + 1));
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (uint32_t *)nullptr, (uint32_t *)nullptr, (int)max_rows);
    void *scan_tmp = nullptr;
    if ((e = cudaMalloc(&scan_tmp, scan_bytes ? scan_bytes : 16)) != cudaSuccess) {
        cudaGetLastError();
        return cleanup(fail(GX_ERR_BAD_MEM_ALLOC, "gx_index_upload: scan scratch"));
    }
    for (int i = 0; i < nlen && e == cudaSuccess; i++) {
        const gx_length_desc &d = lens[i];
        uint32_t *bA_d = ix->bA + (uint64_t)i * nbins;
        if ((e = cudaMemcpy(bA_d, d.bA, sizeof(uint32_t) * nbins, cudaMemcpyHostToDevice)) != cudaSuccess) break;
        if (!d.npep) continue;
        uint32_t *iA_d = ix->iA + hl[i].ia_off;
        const uint64_t nid = (uint64_t)d.npep * d.speclen;
        if ((e = cudaMemcpy(iA_d, d.iA, sizeof(uint32_t) * nid, cudaMemcpyHostToDevice)) != cudaSuccess) break;
        if ((e = cudaMemcpy(ix->mass + hl[i].mass_off, d.mass, sizeof(float) * d.npep, cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            break;
        k_encode_ids<<<(unsigned)std::min<uint64_t>((nid + 255) / 256, 65535), 256>>>(iA_d, nid, d.speclen,
                                                                                    d.speclen / 2, hl[i].magic);
        count_launch();
        uint32_t *blk = ix->blkA + hl[i].blk_off;
        const unsigned g = (nbins + 1 + 255) / 256;
        k_blk_count<<<g, 256>>>(iA_d, bA_d, nbins, E, hl[i].nblk, blk);
        count_launch();
        const int rows = (int)((uint64_t)hl[i].nblk * (nbins + 1));
        size_t tb = scan_bytes;
        if ((e = cub::DeviceScan::ExclusiveSum(scan_tmp, tb, blk, blk, rows)) != cudaSuccess) break;
        count_launch();
        k_blk_scatter<<<g, 256>>>(iA_d, bA_d, blk, nbins, E, hl[i].nblk, ix->iAb + hl[i].ia_off);
        count_launch();
        if ((e = cudaGetLastError()) != cudaSuccess) break;
    }
    cudaFree(scan_tmp);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "gx_index_upload"));
    if ((e = cudaMemcpy(ix->lens, hl.data(), sizeof(DevLen) * nlen, cudaMemcpyHostToDevice)) != cudaSuccess)
        return cleanup(cuda_fail(e, "gx_index_upload lens"));
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return cleanup(cuda_fail(e, "gx_index_upload"));
    *out = ix;
    return GX_SUCCESS;
}
