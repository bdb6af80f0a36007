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

}  // namespace gx
