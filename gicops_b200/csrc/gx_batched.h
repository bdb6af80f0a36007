// Host-side entry points of the batched query path (gx_batched.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "gx_device.cuh"

namespace gx {

// Scratch the batched path needs beyond SearchArgs.
struct BatchedScratch {
    uint64_t *key_in, *key_out;   // scan volume per spectrum (sort keys)
    uint32_t *ord_in, *ord_out;   // spectrum ids
    void *sort_temp;
    size_t sort_temp_bytes;
    int sms;                      // SMs of the device
    int max_ctas[4];              // resident CTAs per SM of k_search_batched<c>, c = 1..3
    bool piped_ok[4];             // k_search_piped<c> fits an SM
};

// Launch shape of the batched path, chosen per workspace (gx_tiles of the C ABI).
struct BatchedTiles {
    int chunks = 2;               // 16-byte id chunks per lane per work unit, 1..3
    int ctas_per_sm = 2;          // persistent CTAs per SM, 1..2 (at most what fits)
    int tile = 0;                 // candidates per scorecard tile (0: the index's block)
    int sorted = 1;               // 1: spectra heaviest first; 0: batch order
    int pipeline = 0;             // 1: k_search_piped (one CTA of 32 warps per SM, two scorecard tiles)
                                  // for the spectra it takes, k_search_batched for the rest
};
constexpr int kMinTile = 1024;

size_t batched_sort_temp_bytes(uint32_t max_spec);
// log10(x) for x in [0, n), computed on the device by the function the kernels call
cudaError_t fill_logtab(double *tab, uint32_t n, cudaStream_t st);
constexpr uint32_t kLogTab = 1u << 20;
cudaError_t batched_set_attributes(int tile);
int batched_ctas_per_sm(int tile, int chunks);   // after batched_set_attributes
uint32_t batched_spill_per_warp(int tile);
bool batched_tiles_valid(const BatchedTiles &t, int max_tile);
bool piped_fits(int tile, int chunks);   // one CTA of the pipelined kernel fits an SM (sets its attributes)
cudaError_t launch_batched(SearchArgs a, const BatchedScratch &b, const BatchedTiles &t, cudaStream_t st);

}  // namespace gx
