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
    int grid;                     // persistent CTAs
};

size_t batched_sort_temp_bytes(uint32_t max_spec);
// log10(x) for x in [0, n), computed on the device by the function the kernels call
cudaError_t fill_logtab(double *tab, uint32_t n, cudaStream_t st);
constexpr uint32_t kLogTab = 1u << 20;
cudaError_t batched_set_attributes(int tile);
int batched_ctas_per_sm(int tile);   // after batched_set_attributes
uint32_t batched_spill_per_warp(int tile);
cudaError_t launch_batched(SearchArgs a, const BatchedScratch &b, cudaStream_t st);

}  // namespace gx
