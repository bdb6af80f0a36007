// Device-resident index (opaque gx_index of the C ABI).
#pragma once

#include <cstdint>
#include <vector>

#include "gx_device.cuh"

namespace gx {
// Entries per block of the block layout; the batched path's scorecard holds one block
// (8 bytes per entry) and block-local ids 2*entry + 1 must fit 16 bits.
#ifndef GX_BLOCK_ENTRIES
#define GX_BLOCK_ENTRIES 11264
#endif
constexpr int kBlockEntries = GX_BLOCK_ENTRIES;
static_assert(2 * kBlockEntries <= 65536 && kBlockEntries % 32 == 0, "block size");
}  // namespace gx

struct gx_index {
    int device = 0;
    int32_t nlen = 0;
    uint32_t nbins = 0;
    uint32_t maxz = 0;
    uint32_t block = gx::kBlockEntries;
    uint32_t *bA = nullptr;    // [nlen][nbins] bin-major CSR offsets (the reference's bA)
    uint32_t *iA = nullptr;    // bin-major ion ids, device form 2*entry + (y ion)
    uint16_t *iAb = nullptr;   // the same ids in block layout, 16-bit block-local
    uint64_t iab_bytes = 0;    // bytes of ids in iAb (the allocation adds one 16-byte chunk)
    uint32_t *blkA = nullptr;  // block layout offsets
    float *mass = nullptr;
    gx::DevLen *lens = nullptr;
    std::vector<gx::DevLen> hlens;
    uint64_t bytes = 0;
};
