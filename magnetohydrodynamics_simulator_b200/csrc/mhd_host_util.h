// Host-side helpers shared by the C-ABI translation units: CUDA error -> mhd_status mapping and
// an early-return macro for CUDA calls.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

#include "../../include/mhd_b200.h"

namespace mhd_host {

inline mhd_status cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return MHD_OK;
    if (e == cudaErrorMemoryAllocation) return MHD_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ||
        e == cudaErrorNoKernelImageForDevice)
        return MHD_ERR_NO_DEVICE;
    return MHD_ERR_CUDA;
}

inline int env_int(const char* name, int def) {
    const char* v = getenv(name);
    return v ? atoi(v) : def;
}

}  // namespace mhd_host

#define MHD_TRY(expr)                                   \
    do {                                                \
        cudaError_t _e = (expr);                        \
        if (_e != cudaSuccess) {                        \
            if (getenv("MHD_B200_VERBOSE"))             \
                fprintf(stderr, "mhd_b200: %s: %s\n", #expr, cudaGetErrorString(_e)); \
            return mhd_host::cuda_status(_e);           \
        }                                               \
    } while (0)
