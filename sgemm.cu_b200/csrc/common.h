// common.h — host-side helpers shared by every translation unit of the library.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "../../include/sgemm_b200.h"

namespace sgb {

// Per-thread status of the most recent public call (sgemm() returns void,
// like the reference, so its outcome is kept here).
void set_last_status(int s);

// Device address of the library's status word (bounded waits write
// SGEMM_B200_ERR_TIMEOUT there).  Resolved once per device.
int* device_status_ptr();

// Cached properties of the current device.
struct DeviceInfo {
    int device = -1;
    int sm_count = 0;
    int cc_major = 0, cc_minor = 0;
    size_t smem_optin = 0;
    char name[256] = {0};
};
const DeviceInfo& device_info();

// True when the current device can run sm_100a code.
bool device_is_sm100();

inline cudaStream_t as_stream(sgemm_b200_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// Detail of the most recent failure on this thread (read back through
// sgemm_b200_last_error_detail): printf-style message.
void note_error(const char* fmt, ...);

inline int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return SGEMM_B200_OK;
    note_error("%s: %s", cudaGetErrorName(e), cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return SGEMM_B200_ERR_NO_MEMORY;
    return SGEMM_B200_ERR_CUDA;
}

// Tensor-map encoding through the driver entry point (no link against libcuda).
bool encode_tensor_map_2d(CUtensorMap* map, CUtensorMapDataType dtype, const void* base,
                          uint64_t inner_elems, uint64_t outer_elems, uint64_t row_stride_bytes,
                          uint32_t box_inner, uint32_t box_outer, CUtensorMapSwizzle swizzle);

// 3-D variant: dims {inner, mid, outer}, byte strides of mid and outer.
bool encode_tensor_map_3d(CUtensorMap* map, CUtensorMapDataType dtype, const void* base,
                          uint64_t inner, uint64_t mid, uint64_t outer, uint64_t mid_stride_bytes,
                          uint64_t outer_stride_bytes, uint32_t box_inner, uint32_t box_mid,
                          uint32_t box_outer, CUtensorMapSwizzle swizzle);

// Library-owned stream-ordered memory pool of the current device, for
// scratch the library allocates itself (split-path workspaces when the caller
// passes none, packed copies of unaligned operands).  Its release threshold is
// unlimited, so freed blocks are reused by the next call instead of going back
// to the driver; the caller's default pool is left untouched.
cudaMemPool_t library_pool();
// The current device's library pool if a call has created it, else null
// (never creates it).
cudaMemPool_t library_pool_if_created();

// Shape checks common to every entry point.  Returns SGEMM_B200_OK or
// SGEMM_B200_ERR_INVALID_ARG.
int check_gemm_args(int m, int n, int k, const float* alpha, const void* A, int lda,
                    const void* B, int ldb, const float* beta, const void* C, int ldc);

inline int div_up(int a, int b) { return (a + b - 1) / b; }

}  // namespace sgb
