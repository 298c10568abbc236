// Host-side helpers shared by the C-ABI translation units: CUDA error -> mhd_status mapping, an
// early-return macro for CUDA calls, and NVTX ranges around the entry points.
#pragma once

#include <cuda_runtime.h>
#ifndef MHD_NO_NVTX
#include <nvtx3/nvToolsExt.h>
#endif

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

// An NVTX range over one entry point's host work (what it enqueues shows under it in a timeline
// or in `ncu --nvtx --nvtx-include "<name>/"`). Header-only NVTX: without a tool attached a push
// and a pop cost a few nanoseconds. Build with -DMHD_NO_NVTX to compile them out.
struct NvtxRange {
    explicit NvtxRange(const char* name) {
#ifndef MHD_NO_NVTX
        nvtxRangePushA(name);
#else
        (void)name;
#endif
    }
    ~NvtxRange() {
#ifndef MHD_NO_NVTX
        nvtxRangePop();
#endif
    }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

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

#define MHD_NVTX_RANGE(name) mhd_host::NvtxRange mhd_nvtx_range_(name)
