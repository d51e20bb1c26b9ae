// common.cu — status word, device cache, tensor-map encoding, argument checks,
// and the small public utility entry points.
#include <cstdarg>
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>

#include "common.h"

namespace sgb {

// The status word bounded device-side waits write into on expiry.
__device__ int g_device_status = 0;

static thread_local int t_last_status = SGEMM_B200_OK;

void set_last_status(int s) { t_last_status = s; }

static constexpr int kMaxDevices = 64;

int* device_status_ptr() {
    static int* ptrs[kMaxDevices] = {nullptr};
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!ptrs[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_device_status) != cudaSuccess) return nullptr;
        ptrs[dev] = static_cast<int*>(p);
    }
    return ptrs[dev];
}

const DeviceInfo& device_info() {
    static DeviceInfo infos[kMaxDevices];
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        static DeviceInfo none;
        return none;
    }
    std::lock_guard<std::mutex> lock(mu);
    DeviceInfo& d = infos[dev];
    if (d.device < 0) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
            d.device = dev;
            d.sm_count = prop.multiProcessorCount;
            d.cc_major = prop.major;
            d.cc_minor = prop.minor;
            d.smem_optin = prop.sharedMemPerBlockOptin;
            std::snprintf(d.name, sizeof(d.name), "%s", prop.name);
        }
    }
    return d;
}

bool device_is_sm100() {
    const DeviceInfo& d = device_info();
    return d.device >= 0 && d.cc_major == 10 && d.cc_minor == 0;
}

static PFN_cuTensorMapEncodeTiled_v12000 get_encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        }
    });
    return fn;
}

bool encode_tensor_map_2d(CUtensorMap* map, CUtensorMapDataType dtype, const void* base,
                          uint64_t inner_elems, uint64_t outer_elems, uint64_t row_stride_bytes,
                          uint32_t box_inner, uint32_t box_outer, CUtensorMapSwizzle swizzle) {
    auto fn = get_encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {inner_elems, outer_elems};
    cuuint64_t strides[1] = {row_stride_bytes};
    cuuint32_t box[2] = {box_inner, box_outer};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, dtype, 2, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        note_error("cuTensorMapEncodeTiled (2-D) returned %d: dims %llu x %llu, row %llu B, "
                   "box %u x %u", (int)r, (unsigned long long)inner_elems,
                   (unsigned long long)outer_elems, (unsigned long long)row_stride_bytes,
                   box_inner, box_outer);
    return r == CUDA_SUCCESS;
}

bool encode_tensor_map_3d(CUtensorMap* map, CUtensorMapDataType dtype, const void* base,
                          uint64_t inner, uint64_t mid, uint64_t outer, uint64_t mid_stride_bytes,
                          uint64_t outer_stride_bytes, uint32_t box_inner, uint32_t box_mid,
                          uint32_t box_outer, CUtensorMapSwizzle swizzle) {
    auto fn = get_encode_fn();
    if (!fn) return false;
    cuuint64_t dims[3] = {inner, mid, outer};
    cuuint64_t strides[2] = {mid_stride_bytes, outer_stride_bytes};
    cuuint32_t box[3] = {box_inner, box_mid, box_outer};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, dtype, 3, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        note_error("cuTensorMapEncodeTiled (3-D) returned %d: dims %llu x %llu x %llu, "
                   "strides %llu %llu B, box %u x %u x %u, base %p", (int)r,
                   (unsigned long long)inner, (unsigned long long)mid, (unsigned long long)outer,
                   (unsigned long long)mid_stride_bytes, (unsigned long long)outer_stride_bytes,
                   box_inner, box_mid, box_outer, base);
    return r == CUDA_SUCCESS;
}

static cudaMemPool_t g_pools[kMaxDevices] = {nullptr};
static std::mutex g_pools_mu;

cudaMemPool_t library_pool_if_created() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(g_pools_mu);
    return g_pools[dev];
}

cudaMemPool_t library_pool() {
    cudaMemPool_t* pools = g_pools;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(g_pools_mu);
    if (!pools[dev]) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
        uint64_t threshold = ~0ull;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &threshold);
        pools[dev] = p;
    }
    return pools[dev];
}

int check_gemm_args(int m, int n, int k, const float* alpha, const void* A, int lda,
                    const void* B, int ldb, const float* beta, const void* C, int ldc) {
    if (m < 0 || n < 0 || k < 0) return SGEMM_B200_ERR_INVALID_ARG;
    if (!alpha || !beta) return SGEMM_B200_ERR_INVALID_ARG;
    if (m == 0 || n == 0) return SGEMM_B200_OK;
    if (ldc < n || !C) return SGEMM_B200_ERR_INVALID_ARG;
    if (k > 0) {
        if (lda < k || ldb < n || !A || !B) return SGEMM_B200_ERR_INVALID_ARG;
    }
    // Index arithmetic inside the kernels is 64-bit for addresses, 32-bit for
    // coordinates; refuse shapes whose coordinates would overflow.
    if ((int64_t)m * ldc > ((int64_t)1 << 40) || (int64_t)m * lda > ((int64_t)1 << 40) ||
        (int64_t)k * ldb > ((int64_t)1 << 40))
        return SGEMM_B200_ERR_INVALID_ARG;
    return SGEMM_B200_OK;
}

}  // namespace sgb

// ------------------------------------------------------------ public utils --

extern "C" int sgemm_b200_device_status(void) {
    int* p = sgb::device_status_ptr();
    if (!p) return SGEMM_B200_ERR_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess) return SGEMM_B200_ERR_CUDA;
    int v = 0;
    if (cudaMemcpy(&v, p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SGEMM_B200_ERR_CUDA;
    const int zero = 0;
    if (cudaMemcpy(p, &zero, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
        return SGEMM_B200_ERR_CUDA;
    return v;
}

extern "C" int sgemm_b200_last_status(void) { return sgb::t_last_status; }

extern "C" const char* sgemm_b200_status_string(int s) {
    switch (s) {
        case SGEMM_B200_OK: return "ok";
        case SGEMM_B200_ERR_INVALID_ARG: return "invalid argument";
        case SGEMM_B200_ERR_UNSUPPORTED: return "unsupported device or mode";
        case SGEMM_B200_ERR_CUDA: return "CUDA error";
        case SGEMM_B200_ERR_TIMEOUT: return "device-side wait timed out";
        case SGEMM_B200_ERR_NO_MEMORY: return "out of memory or workspace too small";
        case SGEMM_B200_ERR_REJECTED: return "request rejected by admission control";
        default: return "unknown status";
    }
}

extern "C" const char* sgemm_b200_version(void) { return "sgemm_b200 0.2.0 (sm_100a)"; }

extern "C" int sgemm_b200_abi_version(void) { return SGEMM_B200_ABI_VERSION; }

namespace sgb {
static thread_local char g_error_detail[512] = "";
void note_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_error_detail, sizeof(g_error_detail), fmt, ap);
    va_end(ap);
}
}  // namespace sgb

extern "C" const char* sgemm_b200_last_error_detail(void) { return sgb::g_error_detail; }

extern "C" int sgemm_b200_pool_usage(size_t* used_bytes, size_t* reserved_bytes) {
    if (!used_bytes || !reserved_bytes) return SGEMM_B200_ERR_INVALID_ARG;
    *used_bytes = *reserved_bytes = 0;
    cudaMemPool_t p = sgb::library_pool_if_created();  // never creates the pool
    if (!p) return SGEMM_B200_OK;
    uint64_t used = 0, reserved = 0;
    cudaError_t e = cudaMemPoolGetAttribute(p, cudaMemPoolAttrUsedMemCurrent, &used);
    if (e == cudaSuccess) e = cudaMemPoolGetAttribute(p, cudaMemPoolAttrReservedMemCurrent, &reserved);
    if (e != cudaSuccess) return sgb::cuda_status(e);
    *used_bytes = (size_t)used;
    *reserved_bytes = (size_t)reserved;
    return SGEMM_B200_OK;
}
