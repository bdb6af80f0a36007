// Scoped switch of the calling host thread's current CUDA device.
#pragma once

#include <cuda_runtime.h>

namespace gx {

// Makes `device` current for the lifetime of the object and makes the caller's device
// current again when it ends, so that an entry point never leaves a host thread that
// drives several GPUs on another device than the one it called with.  status() is the
// result of the switch (cudaSuccess when the device was already current).
class DeviceScope {
public:
    explicit DeviceScope(int device)
    {
        if (cudaGetDevice(&prev_) != cudaSuccess) {
            cudaGetLastError();
            prev_ = -1;
        }
        if (prev_ == device) return;
        err_ = cudaSetDevice(device);
        switched_ = err_ == cudaSuccess && prev_ >= 0;
    }
    ~DeviceScope()
    {
        if (switched_) cudaSetDevice(prev_);
    }
    DeviceScope(const DeviceScope &) = delete;
    DeviceScope &operator=(const DeviceScope &) = delete;
    cudaError_t status() const { return err_; }

private:
    int prev_ = -1;
    bool switched_ = false;
    cudaError_t err_ = cudaSuccess;
};

}  // namespace gx
