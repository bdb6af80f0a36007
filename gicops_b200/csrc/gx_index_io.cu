// Device index to and from a file.
//
// The reference rebuilds its index in every run and caches only preprocessed spectra
// (source/core/msquery.cpp:542-721).  The index of the large configuration (27 GB in HBM,
// 20 s to build from host arrays) is worth keeping: gx_index_save writes every device array as
// the device holds it (bin offsets, re-encoded ids, the block layout, masses, per-length
// constants) and gx_index_load puts them back on a device without building anything.
//
// File layout (little-endian): magic "GXIDX001"; uint32 nlen, nbins, maxz, block,
// sizeof(DevLen), 0; uint64 tot_ia, tot_m, tot_blk, total file bytes; DevLen[nlen]; then
// bA [nlen * nbins] u32, iA [tot_ia] u32, iAb [tot_ia] u16, blkA [tot_blk] u32, mass [tot_m]
// f32.  Arrays travel through one pinned staging buffer of at most kStage bytes.

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/gicops_b200.h"
#include "gx_device_scope.cuh"
#include "gx_index.cuh"
#include "gx_internal.h"

using namespace gx;

namespace {

constexpr char kMagic[8] = {'G', 'X', 'I', 'D', 'X', '0', '0', '1'};
constexpr size_t kStage = 64ull << 20;

struct Header {
    char magic[8];
    uint32_t nlen, nbins, maxz, block, devlen_bytes, pad;
    uint64_t tot_ia, tot_m, tot_blk, file_bytes;
};
static_assert(sizeof(Header) == 64, "index file header");

struct File {
    FILE *f = nullptr;
    ~File()
    {
        if (f) std::fclose(f);
    }
};

struct Pinned {
    void *p = nullptr;
    ~Pinned()
    {
        if (p) cudaFreeHost(p);
    }
};

void totals(const gx_index *ix, uint64_t &tot_ia, uint64_t &tot_m, uint64_t &tot_blk)
{
    tot_ia = tot_m = tot_blk = 0;
    for (const DevLen &l : ix->hlens) {
        tot_ia = std::max<uint64_t>(tot_ia, l.ia_off + (uint64_t)l.npep * l.speclen);
        tot_m = std::max<uint64_t>(tot_m, l.mass_off + l.npep);
        tot_blk = std::max<uint64_t>(tot_blk, l.blk_off + (uint64_t)l.nblk * (ix->nbins + 1));
    }
}

// device array <-> file through the staging buffer
gx_status dump(FILE *f, const void *dev, uint64_t bytes, void *stage, const char *what)
{
    for (uint64_t o = 0; o < bytes; o += kStage) {
        const size_t n = (size_t)std::min<uint64_t>(kStage, bytes - o);
        cudaError_t e = cudaMemcpy(stage, static_cast<const char *>(dev) + o, n, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, what);
        if (std::fwrite(stage, 1, n, f) != n) return fail(GX_ERR_INVLD_MEMORY, std::string(what) + ": write failed");
    }
    return GX_SUCCESS;
}

gx_status fill(FILE *f, void *dev, uint64_t bytes, void *stage, const char *what)
{
    for (uint64_t o = 0; o < bytes; o += kStage) {
        const size_t n = (size_t)std::min<uint64_t>(kStage, bytes - o);
        if (std::fread(stage, 1, n, f) != n) return fail(GX_ERR_NOT_ENOUGH_DATA, std::string(what) + ": file too short");
        cudaError_t e = cudaMemcpy(static_cast<char *>(dev) + o, stage, n, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, what);
    }
    return GX_SUCCESS;
}

}  // namespace

extern "C" gx_status gx_index_save(const gx_index *ix, const char *path)
{
    if (!ix || !path) return fail(GX_ERR_INVLD_PTR, "gx_index_save: null argument");
    uint64_t tot_ia, tot_m, tot_blk;
    totals(ix, tot_ia, tot_m, tot_blk);
    Header h{};
    std::memcpy(h.magic, kMagic, 8);
    h.nlen = (uint32_t)ix->nlen;
    h.nbins = ix->nbins;
    h.maxz = ix->maxz;
    h.block = ix->block;
    h.devlen_bytes = (uint32_t)sizeof(DevLen);
    h.tot_ia = tot_ia;
    h.tot_m = tot_m;
    h.tot_blk = tot_blk;
    h.file_bytes = sizeof(Header) + sizeof(DevLen) * (uint64_t)ix->nlen + 4ull * ix->nbins * ix->nlen + 4 * tot_ia +
                   2 * tot_ia + 4 * tot_blk + 4 * tot_m;
    File fh;
    fh.f = std::fopen(path, "wb");
    if (!fh.f) return fail(GX_ERR_FILE_NOT_FOUND, std::string("gx_index_save: cannot open ") + path);
    DeviceScope ds(ix->device);
    if (ds.status() != cudaSuccess) return cuda_fail(ds.status(), "gx_index_save: cudaSetDevice");
    cudaGetLastError();
    Pinned stage;
    cudaError_t e = cudaMallocHost(&stage.p, kStage);
    if (e != cudaSuccess) return cuda_fail(e, "gx_index_save: staging buffer");
    if (std::fwrite(&h, sizeof(h), 1, fh.f) != 1 ||
        std::fwrite(ix->hlens.data(), sizeof(DevLen), (size_t)ix->nlen, fh.f) != (size_t)ix->nlen)
        return fail(GX_ERR_INVLD_MEMORY, "gx_index_save: write failed");
    gx_status st;
    if ((st = dump(fh.f, ix->bA, 4ull * ix->nbins * ix->nlen, stage.p, "gx_index_save: bA")) != GX_SUCCESS ||
        (st = dump(fh.f, ix->iA, 4 * tot_ia, stage.p, "gx_index_save: iA")) != GX_SUCCESS ||
        (st = dump(fh.f, ix->iAb, 2 * tot_ia, stage.p, "gx_index_save: iAb")) != GX_SUCCESS ||
        (st = dump(fh.f, ix->blkA, 4 * tot_blk, stage.p, "gx_index_save: blkA")) != GX_SUCCESS ||
        (st = dump(fh.f, ix->mass, 4 * tot_m, stage.p, "gx_index_save: mass")) != GX_SUCCESS)
        return st;
    if (std::fflush(fh.f) != 0) return fail(GX_ERR_INVLD_MEMORY, "gx_index_save: write failed");
    return GX_SUCCESS;
}

extern "C" gx_status gx_index_load(const char *path, int32_t device, gx_index **out)
{
    if (!path || !out) return fail(GX_ERR_INVLD_PTR, "gx_index_load: null argument");
    *out = nullptr;
    File fh;
    fh.f = std::fopen(path, "rb");
    if (!fh.f) return fail(GX_ERR_FILE_NOT_FOUND, std::string("gx_index_load: cannot open ") + path);
    Header h{};
    if (std::fread(&h, sizeof(h), 1, fh.f) != 1 || std::memcmp(h.magic, kMagic, 8) != 0)
        return fail(GX_ERR_INVLD_INDEX, "gx_index_load: not an index file of this library");
    if (h.devlen_bytes != sizeof(DevLen) || h.nlen < 1 || h.nlen > GX_MAX_LENGTHS || h.nbins < 2)
        return fail(GX_ERR_INVLD_INDEX, "gx_index_load: header does not match this library's layout");
    if (h.block != (uint32_t)kBlockEntries)
        return fail(GX_ERR_INVLD_INDEX, "gx_index_load: the file's entry block (" + std::to_string(h.block) +
                                            ") differs from this library's (" + std::to_string(kBlockEntries) + ")");
    std::vector<DevLen> hl(h.nlen);
    if (std::fread(hl.data(), sizeof(DevLen), h.nlen, fh.f) != h.nlen)
        return fail(GX_ERR_NOT_ENOUGH_DATA, "gx_index_load: file too short");
    if (std::fseek(fh.f, 0, SEEK_END) != 0 || (uint64_t)std::ftell(fh.f) != h.file_bytes ||
        std::fseek(fh.f, (long)(sizeof(Header) + sizeof(DevLen) * h.nlen), SEEK_SET) != 0)
        return fail(GX_ERR_NOT_ENOUGH_DATA, "gx_index_load: file size does not match its header");
    DeviceScope ds(device);
    if (ds.status() != cudaSuccess) return cuda_fail(ds.status(), "gx_index_load: cudaSetDevice");
    cudaGetLastError();
    auto *ix = new gx_index();
    ix->device = device;
    ix->nlen = (int32_t)h.nlen;
    ix->nbins = h.nbins;
    ix->maxz = h.maxz;
    ix->block = h.block;
    ix->hlens = hl;
    const uint64_t tot_ia = h.tot_ia, tot_m = h.tot_m, tot_blk = h.tot_blk;
    cudaError_t e;
    if ((e = cudaMalloc(&ix->bA, 4ull * h.nbins * h.nlen)) != cudaSuccess ||
        (e = cudaMalloc(&ix->iA, 4 * (tot_ia ? tot_ia : 1))) != cudaSuccess ||
        (e = cudaMalloc(&ix->iAb, 2 * (tot_ia + 8))) != cudaSuccess ||
        (e = cudaMalloc(&ix->blkA, 4 * (tot_blk ? tot_blk : 1))) != cudaSuccess ||
        (e = cudaMalloc(&ix->mass, 4 * (tot_m ? tot_m : 1))) != cudaSuccess ||
        (e = cudaMalloc(&ix->lens, sizeof(DevLen) * h.nlen)) != cudaSuccess ||
        (e = cudaMemset(ix->iAb + tot_ia, 0, 8 * sizeof(uint16_t))) != cudaSuccess) {
        cudaGetLastError();
        gx_index_free(ix);
        return fail(GX_ERR_BAD_MEM_ALLOC, std::string("gx_index_load: ") + cudaGetErrorString(e));
    }
    ix->bytes = 4 * ((uint64_t)h.nbins * h.nlen + tot_ia + tot_blk) + 2 * (tot_ia + 8) + 4 * tot_m +
                sizeof(DevLen) * h.nlen;
    ix->iab_bytes = 2 * tot_ia;
    Pinned stage;
    gx_status st = GX_SUCCESS;
    if ((e = cudaMallocHost(&stage.p, kStage)) != cudaSuccess) st = cuda_fail(e, "gx_index_load: staging buffer");
    if (st == GX_SUCCESS) st = fill(fh.f, ix->bA, 4ull * h.nbins * h.nlen, stage.p, "gx_index_load: bA");
    if (st == GX_SUCCESS) st = fill(fh.f, ix->iA, 4 * tot_ia, stage.p, "gx_index_load: iA");
    if (st == GX_SUCCESS) st = fill(fh.f, ix->iAb, 2 * tot_ia, stage.p, "gx_index_load: iAb");
    if (st == GX_SUCCESS) st = fill(fh.f, ix->blkA, 4 * tot_blk, stage.p, "gx_index_load: blkA");
    if (st == GX_SUCCESS) st = fill(fh.f, ix->mass, 4 * tot_m, stage.p, "gx_index_load: mass");
    if (st == GX_SUCCESS && (e = cudaMemcpy(ix->lens, hl.data(), sizeof(DevLen) * h.nlen, cudaMemcpyHostToDevice)) !=
                                cudaSuccess)
        st = cuda_fail(e, "gx_index_load: lengths");
    if (st != GX_SUCCESS) {
        gx_index_free(ix);
        return st;
    }
    *out = ix;
    return GX_SUCCESS;
}
