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
#include "gx_device_scope.cuh"
#include "gx_internal.h"
#include "gx_ions.h"

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
    DeviceScope ds(ix->device);
    cudaFree(ix->bA);
    cudaFree(ix->iA);
    cudaFree(ix->iAb);
    cudaFree(ix->blkA);
    cudaFree(ix->mass);
    cudaFree(ix->lens);
    delete ix;
    cudaGetLastError();   // nothing of a free is reported to the next call
    return GX_SUCCESS;
}

extern "C" uint64_t gx_index_bytes(const gx_index *ix) { return ix ? ix->bytes : 0; }

namespace {

// Allocates the index arrays for the lengths `hl` (offsets already set) and the scan
// scratch of the block layout.
gx_status alloc_index(std::vector<DevLen> &hl, int32_t nlen, uint32_t nbins, uint32_t maxz, uint64_t tot_ia,
                      uint64_t tot_m, uint64_t tot_blk, int32_t device, gx_index **out, void **scan_tmp,
                      size_t *scan_bytes, const char *who)
{
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, (std::string(who) + ": cudaSetDevice").c_str());
    auto *ix = new gx_index();
    ix->device = device;
    ix->nlen = nlen;
    ix->nbins = nbins;
    ix->maxz = maxz;
    ix->block = (uint32_t)kBlockEntries;
    ix->hlens = hl;
    if ((e = cudaMalloc(&ix->bA, sizeof(uint32_t) * (uint64_t)nbins * nlen)) != cudaSuccess ||
        (e = cudaMalloc(&ix->iA, sizeof(uint32_t) * (tot_ia ? tot_ia : 1))) != cudaSuccess ||
        (e = cudaMalloc(&ix->iAb, sizeof(uint16_t) * (tot_ia + 8))) != cudaSuccess ||
        (e = cudaMalloc(&ix->blkA, sizeof(uint32_t) * (tot_blk ? tot_blk : 1))) != cudaSuccess ||
        (e = cudaMalloc(&ix->mass, sizeof(float) * (tot_m ? tot_m : 1))) != cudaSuccess ||
        (e = cudaMalloc(&ix->lens, sizeof(DevLen) * nlen)) != cudaSuccess) {
        cudaGetLastError();
        gx_index_free(ix);
        return fail(GX_ERR_BAD_MEM_ALLOC, std::string(who) + ": " + cudaGetErrorString(e));
    }
    ix->bytes = sizeof(uint32_t) * ((uint64_t)nbins * nlen + tot_ia + tot_blk) + sizeof(uint16_t) * (tot_ia + 8) +
                sizeof(float) * tot_m + sizeof(DevLen) * nlen;
    ix->iab_bytes = sizeof(uint16_t) * tot_ia;
    if ((e = cudaMemset(ix->iAb + tot_ia, 0, 8 * sizeof(uint16_t))) != cudaSuccess) {
        gx_index_free(ix);
        return cuda_fail(e, (std::string(who) + ": iAb padding").c_str());
    }
    // scan scratch, sized for the largest per-length offset table
    uint64_t max_rows = 1;
    for (int i = 0; i < nlen; i++) max_rows = std::max<uint64_t>(max_rows, (uint64_t)hl[i].nblk * (nbins + 1));
    *scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, *scan_bytes, (uint32_t *)nullptr, (uint32_t *)nullptr, (int)max_rows);
    if ((e = cudaMalloc(scan_tmp, *scan_bytes ? *scan_bytes : 16)) != cudaSuccess) {
        cudaGetLastError();
        gx_index_free(ix);
        return fail(GX_ERR_BAD_MEM_ALLOC, std::string(who) + ": scan scratch");
    }
    *out = ix;
    return GX_SUCCESS;
}

// Device forms of length i from its bin-major arrays already in ix->bA / ix->iA (raw ids
// entry*speclen + pos): ids re-encoded as 2*entry + (y ion), then the block layout.
cudaError_t finish_length(gx_index *ix, int i, void *scan_tmp, size_t scan_bytes)
{
    const DevLen &l = ix->hlens[i];
    if (!l.npep) return cudaSuccess;
    const uint32_t nbins = ix->nbins, E = ix->block;
    uint32_t *bA_d = ix->bA + (uint64_t)i * nbins;
    uint32_t *iA_d = ix->iA + l.ia_off;
    const uint64_t nid = (uint64_t)l.npep * l.speclen;
    k_encode_ids<<<(unsigned)std::min<uint64_t>((nid + 255) / 256, 65535), 256>>>(iA_d, nid, l.speclen, l.half, l.magic);
    count_launch();
    uint32_t *blk = ix->blkA + l.blk_off;
    const unsigned g = (nbins + 1 + 255) / 256;
    k_blk_count<<<g, 256>>>(iA_d, bA_d, nbins, E, l.nblk, blk);
    count_launch();
    const int rows = (int)((uint64_t)l.nblk * (nbins + 1));
    size_t tb = scan_bytes;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(scan_tmp, tb, blk, blk, rows);
    if (e != cudaSuccess) return e;
    count_launch();
    k_blk_scatter<<<g, 256>>>(iA_d, bA_d, blk, nbins, E, l.nblk, ix->iAb + l.ia_off);
    count_launch();
    return cudaGetLastError();
}

gx_status finish_index(gx_index *ix, const char *who)
{
    cudaError_t e;
    if ((e = cudaMemcpy(ix->lens, ix->hlens.data(), sizeof(DevLen) * ix->nlen, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaDeviceSynchronize()) != cudaSuccess) {
        gx_index_free(ix);
        return cuda_fail(e, who);
    }
    return GX_SUCCESS;
}

DevLen dev_len(uint32_t npep, uint32_t speclen, uint32_t peplen, uint64_t ia_off, uint64_t mass_off, uint64_t blk_off)
{
    const uint32_t E = (uint32_t)kBlockEntries;
    const uint32_t magic = (uint32_t)(((1ull << 32) + speclen - 1) / speclen);
    const uint32_t nblk = npep ? (npep + E - 1) / E : 0;
    return DevLen{ia_off, mass_off, npep, speclen, speclen / 2, peplen, magic, nblk, blk_off};
}

}  // namespace

extern "C" gx_status gx_index_upload(const gx_length_desc *lens, int32_t nlen, uint32_t nbins, int32_t device,
                                     gx_index **out)
{
    if (!lens || !out) return fail(GX_ERR_INVLD_PTR, "gx_index_upload: null argument");
    *out = nullptr;
    if (nlen < 1 || nlen > GX_MAX_LENGTHS || nbins < 2)
        return fail(GX_ERR_INVLD_PARAM, "gx_index_upload: nlen must be 1..64 and nbins >= 2");
    cudaGetLastError();   // an earlier call's error is not ours to report
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
        hl[i] = dev_len(d.npep, d.speclen, d.peplen, tot_ia, tot_m, tot_blk);
        tot_ia += (uint64_t)d.npep * d.speclen;
        tot_m += d.npep;
        tot_blk += (uint64_t)hl[i].nblk * (nbins + 1);
    }
    gx_index *ix = nullptr;
    void *scan_tmp = nullptr;
    size_t scan_bytes = 0;
    DeviceScope ds(device);   // the caller's device is current again on return
    gx_status st = alloc_index(hl, nlen, nbins, maxz, tot_ia, tot_m, tot_blk, device, &ix, &scan_tmp, &scan_bytes,
                               "gx_index_upload");
    if (st != GX_SUCCESS) return st;
    cudaError_t e = cudaSuccess;
    const char *step = "";
    for (int i = 0; i < nlen && e == cudaSuccess; i++) {
        const gx_length_desc &d = lens[i];
        step = "gx_index_upload: bA copy";
        if ((e = cudaMemcpy(ix->bA + (uint64_t)i * nbins, d.bA, sizeof(uint32_t) * nbins, cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            break;
        if (!d.npep) continue;
        const uint64_t nid = (uint64_t)d.npep * d.speclen;
        step = "gx_index_upload: iA / mass copy";
        if ((e = cudaMemcpy(ix->iA + hl[i].ia_off, d.iA, sizeof(uint32_t) * nid, cudaMemcpyHostToDevice)) !=
                cudaSuccess ||
            (e = cudaMemcpy(ix->mass + hl[i].mass_off, d.mass, sizeof(float) * d.npep, cudaMemcpyHostToDevice)) !=
                cudaSuccess)
            break;
        step = "gx_index_upload: id encoding / block layout";
        e = finish_length(ix, i, scan_tmp, scan_bytes);
    }
    cudaFree(scan_tmp);
    if (e != cudaSuccess) {
        gx_index_free(ix);
        return cuda_fail(e, step);
    }
    if ((st = finish_index(ix, "gx_index_upload")) != GX_SUCCESS) return st;
    *out = ix;
    return GX_SUCCESS;
}

// ------------------------------------------------------------------------------------
// Device index builder: the ion / CSR stage of the build (the reference's
// DSLIM_Construct, source/core/dslim.cpp:231-504, with the ion arithmetic of
// utils.cpp:161-474) on the GPU, from entries built on the host.  One thread per
// (entry, ion series) writes the series' bins and ids; a stable radix sort by bin
// keeps ids ascending inside a bin, as the reference's counting sort does; bA comes
// from the sorted bins.  The arrays equal those of the host builder.
// ------------------------------------------------------------------------------------
namespace gx {

__global__ void k_ions(const char *__restrict__ seqs, const gx_pep_entry *__restrict__ ent, uint32_t N, uint32_t L,
                       uint32_t maxz, ions::IonTables tab, double minmass, double maxmass, uint32_t topbin,
                       uint32_t *keys, uint32_t *vals)
{
    __shared__ ions::IonTables t;
    for (int w = threadIdx.x; w < (int)(sizeof(ions::IonTables) / 4); w += blockDim.x)
        reinterpret_cast<uint32_t *>(&t)[w] = reinterpret_cast<const uint32_t *>(&tab)[w];
    __syncthreads();
    const uint32_t nser = 2 * maxz, n1 = L - 1, speclen = nser * n1;
    const uint64_t total = (uint64_t)N * nser;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = (uint32_t)(g / nser), s = (uint32_t)(g % nser);
        const bool y = s >= maxz;
        const uint32_t z = y ? s - maxz : s;
        const gx_pep_entry e = ent[k];
        const char *seq = seqs + (uint64_t)e.seqid * L;
        // positions: b ions of charge z at z*(L-1), y ions at (maxz + z)*(L-1)
        const uint64_t id0 = (uint64_t)k * speclen + (uint64_t)(y ? maxz + z : z) * n1;
        if (ions::entry_binned(t, seq, L, e.sites, e.modnum, minmass, maxmass))
            ions::ion_series(t, seq, L, e.sites, e.modnum, z, y, topbin, keys + id0);
        else
            for (uint32_t l = 0; l < n1; l++) keys[id0 + l] = 0;
        for (uint32_t l = 0; l < n1; l++) vals[id0 + l] = (uint32_t)(id0 + l);
    }
}

// bA[b] = number of ids in bins below b, from the bins sorted ascending: the bins
// (key[i-1], key[i]] start at i (key[-1] = -1, key[n] = nbins - 1 past the last).
__global__ void k_bin_offsets(const uint32_t *__restrict__ key, uint32_t n, uint32_t nbins, uint32_t *bA)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t lo = i == 0 ? 0u : key[i - 1] + 1u;
        const uint32_t hi = i == n ? nbins - 1u : key[i];
        for (uint32_t b = lo; b <= hi; b++) bA[b] = (uint32_t)i;
    }
}

__global__ void k_entry_mass(const gx_pep_entry *__restrict__ ent, uint32_t N, float *mass)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < N) mass[k] = ent[k].mass;
}

}  // namespace gx

extern "C" gx_status gx_index_build(gx_host_length *const *lens, int32_t nlen, const gx_build_params *bp,
                                    int32_t device, gx_index **out)
{
    if (!lens || !bp || !out) return fail(GX_ERR_INVLD_PTR, "gx_index_build: null argument");
    *out = nullptr;
    if (nlen < 1 || nlen > GX_MAX_LENGTHS) return fail(GX_ERR_INVLD_PARAM, "gx_index_build: nlen must be 1..64");
    cudaGetLastError();   // an earlier call's error is not ours to report
    if (bp->maxz < 1 || bp->maxz > 6 || bp->scale == 0 || bp->max_mass <= bp->min_mass ||
        bp->nmods > (uint32_t)ions::kMaxModTypes)
        return fail(GX_ERR_INVLD_PARAM, "gx_index_build: bad parameters");
    const uint64_t topbin64 = (uint64_t)bp->max_mass * bp->scale;
    if (topbin64 + 1 >= (1ull << 31)) return fail(GX_ERR_INVLD_PARAM, "gx_index_build: max_mass * scale too large");
    const uint32_t topbin = (uint32_t)topbin64, nbins = topbin + 1;
    struct Src {
        gx_length_desc d;
        const gx_pep_entry *ent;
        const char *seqs;
        uint32_t nkept;
    };
    std::vector<Src> src(nlen);
    std::vector<DevLen> hl(nlen);
    uint64_t tot_ia = 0, tot_m = 0, tot_blk = 0, max_n = 0, max_ent = 0, max_seq = 0;
    for (int i = 0; i < nlen; i++) {
        if (!lens[i]) return fail(GX_ERR_INVLD_PTR, "gx_index_build: null length");
        Src &x = src[i];
        gx_status st = gx_host_length_desc(lens[i], &x.d);
        if (st != GX_SUCCESS) return st;
        x.ent = gx_host_length_entries(lens[i]);
        x.seqs = gx_host_length_seqs(lens[i], &x.nkept);
        const uint32_t L = x.d.peplen;
        if (L < 2 || L > (uint32_t)ions::kMaxSeqLen || x.d.speclen != 2 * (L - 1) * bp->maxz)
            return fail(GX_ERR_INVLD_INDEX, "gx_index_build: length built with another maxz");
        const uint64_t n = (uint64_t)x.d.npep * x.d.speclen;
        if (n >= (1ull << 31)) return fail(GX_ERR_INVLD_SIZE, "gx_index_build: 2^31 or more ion ids in one length");
        if (x.d.npep && (!x.ent || !x.seqs)) return fail(GX_ERR_INVLD_PTR, "gx_index_build: length without entries");
        for (uint32_t k = 0; k < x.d.npep; k++)
            if (x.ent[k].seqid >= x.nkept) return fail(GX_ERR_INVLD_INDEX, "gx_index_build: entry without sequence");
        hl[i] = dev_len(x.d.npep, x.d.speclen, L, tot_ia, tot_m, tot_blk);
        tot_ia += n;
        tot_m += x.d.npep;
        tot_blk += (uint64_t)hl[i].nblk * (nbins + 1);
        max_n = std::max(max_n, n);
        max_ent = std::max<uint64_t>(max_ent, x.d.npep);
        max_seq = std::max<uint64_t>(max_seq, (uint64_t)x.nkept * L);
    }
    gx_index *ix = nullptr;
    void *scan_tmp = nullptr;
    size_t scan_bytes = 0;
    DeviceScope ds(device);   // the caller's device is current again on return
    gx_status st = alloc_index(hl, nlen, nbins, bp->maxz, tot_ia, tot_m, tot_blk, device, &ix, &scan_tmp, &scan_bytes,
                               "gx_index_build");
    if (st != GX_SUCCESS) return st;
    // build scratch, sized for the largest length
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                    (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)std::max<uint64_t>(max_n, 1));
    uint32_t *keys = nullptr, *keys_out = nullptr, *vals = nullptr;
    void *sort_tmp = nullptr;
    char *d_seqs = nullptr;
    gx_pep_entry *d_ent = nullptr;
    cudaError_t e;
    if ((e = cudaMalloc(&keys, sizeof(uint32_t) * std::max<uint64_t>(max_n, 1))) != cudaSuccess ||
        (e = cudaMalloc(&keys_out, sizeof(uint32_t) * std::max<uint64_t>(max_n, 1))) != cudaSuccess ||
        (e = cudaMalloc(&vals, sizeof(uint32_t) * std::max<uint64_t>(max_n, 1))) != cudaSuccess ||
        (e = cudaMalloc(&sort_tmp, sort_bytes ? sort_bytes : 16)) != cudaSuccess ||
        (e = cudaMalloc(&d_seqs, std::max<uint64_t>(max_seq, 1))) != cudaSuccess ||
        (e = cudaMalloc(&d_ent, sizeof(gx_pep_entry) * std::max<uint64_t>(max_ent, 1))) != cudaSuccess)
        cudaGetLastError();
    const ions::IonTables tab = ion_tables(bp);
    const char *step = "gx_index_build: build scratch";
    const int end_bit = 32 - __builtin_clz(topbin);
    for (int i = 0; i < nlen && e == cudaSuccess; i++) {
        const Src &x = src[i];
        uint32_t *bA_d = ix->bA + (uint64_t)i * nbins;
        const uint32_t N = x.d.npep, L = x.d.peplen;
        if (!N) {
            e = cudaMemset(bA_d, 0, sizeof(uint32_t) * nbins);
            continue;
        }
        const uint64_t n = (uint64_t)N * x.d.speclen;
        step = "gx_index_build: entry copy";
        if ((e = cudaMemcpy(d_seqs, x.seqs, (size_t)x.nkept * L, cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(d_ent, x.ent, sizeof(gx_pep_entry) * N, cudaMemcpyHostToDevice)) != cudaSuccess)
            break;
        step = "gx_index_build: ions / sort / offsets";
        const uint64_t threads = (uint64_t)N * 2 * bp->maxz;
        k_ions<<<(unsigned)std::min<uint64_t>((threads + 255) / 256, 1u << 20), 256>>>(
            d_seqs, d_ent, N, L, bp->maxz, tab, (double)bp->min_mass, (double)bp->max_mass, topbin, keys, vals);
        count_launch();
        size_t tb = sort_bytes;
        if ((e = cub::DeviceRadixSort::SortPairs(sort_tmp, tb, keys, keys_out, vals, ix->iA + hl[i].ia_off, (int)n, 0,
                                                 end_bit)) != cudaSuccess)
            break;
        count_launch();
        k_bin_offsets<<<(unsigned)std::min<uint64_t>((n + 1 + 255) / 256, 1u << 20), 256>>>(keys_out, (uint32_t)n,
                                                                                          nbins, bA_d);
        count_launch();
        k_entry_mass<<<(N + 255) / 256, 256>>>(d_ent, N, ix->mass + hl[i].mass_off);
        count_launch();
        if ((e = cudaGetLastError()) != cudaSuccess) break;
        step = "gx_index_build: id encoding / block layout";
        e = finish_length(ix, i, scan_tmp, scan_bytes);
    }
    cudaDeviceSynchronize();
    cudaFree(keys);
    cudaFree(keys_out);
    cudaFree(vals);
    cudaFree(sort_tmp);
    cudaFree(d_seqs);
    cudaFree(d_ent);
    cudaFree(scan_tmp);
    if (e != cudaSuccess) {
        gx_index_free(ix);
        if (e == cudaErrorMemoryAllocation) return fail(GX_ERR_BAD_MEM_ALLOC, "gx_index_build: build scratch");
        return cuda_fail(e, step);
    }
    if ((st = finish_index(ix, "gx_index_build")) != GX_SUCCESS) return st;
    *out = ix;
    return GX_SUCCESS;
}

extern "C" gx_status gx_index_read_length(const gx_index *ix, int32_t i, uint32_t *bA, uint32_t *iA, uint16_t *iAb,
                                          float *mass)
{
    if (!ix) return fail(GX_ERR_INVLD_PTR, "gx_index_read_length: null index");
    if (i < 0 || i >= ix->nlen) return fail(GX_ERR_INVLD_PARAM, "gx_index_read_length: no such length");
    DeviceScope ds(ix->device);
    cudaError_t e = ds.status();
    if (e != cudaSuccess) return cuda_fail(e, "gx_index_read_length: cudaSetDevice");
    const DevLen &l = ix->hlens[i];
    const uint64_t n = (uint64_t)l.npep * l.speclen;
    if (bA && (e = cudaMemcpy(bA, ix->bA + (uint64_t)i * ix->nbins, sizeof(uint32_t) * ix->nbins,
                              cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "gx_index_read_length: bA");
    if (iA && n && (e = cudaMemcpy(iA, ix->iA + l.ia_off, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "gx_index_read_length: iA");
    if (iAb && n &&
        (e = cudaMemcpy(iAb, ix->iAb + l.ia_off, sizeof(uint16_t) * n, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "gx_index_read_length: iAb");
    if (mass && l.npep &&
        (e = cudaMemcpy(mass, ix->mass + l.mass_off, sizeof(float) * l.npep, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "gx_index_read_length: mass");
    return GX_SUCCESS;
}
