// Internal helpers shared by the host sources of libgicops_b200.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/gicops_b200.h"

namespace gx {

// Records `msg` as the calling thread's last error and returns `code`.
gx_status fail(gx_status code, const std::string &msg);

// Records a CUDA failure (message "what: cuda error string") and returns GX_ERR_CUDA.
gx_status cuda_fail(int cuda_error, const char *what);

// Number of kernels launched so far by this library.
void count_launch(uint64_t n = 1);

// Opt-in kernel timing (events on the launching stream); prof_begin returns -1 when off.
int prof_begin(const char *name, void *stream);
void prof_end(int handle, void *stream);

// Search of a batch already in device memory through a workspace, on `stream` (the
// launch sequence of gx_search_device after its argument checks; the index's device must
// be current).  heap / hist may be NULL.
gx_status search_launch(gx_index *ix, gx_workspace *ws, const gx_queries *q_dev, const gx_params *p, gx_result *out,
                        gx_cell *heap, uint32_t *hist, void *stream);
// The workspace's own stream, and its device guard word (device memory, int32).
void *workspace_stream(gx_workspace *ws);
int32_t *workspace_err(gx_workspace *ws);

}  // namespace gx
