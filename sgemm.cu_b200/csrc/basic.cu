// basic.cu — the naive kernel (one thread per C element) and the seeded
// counter-based generator used by the harnesses.
//
// sgemm_b200_basic replaces sgemm_basic()/kernel_basic
// (src/sgemm.cuh:92-113, src/kernels/basic.cuh:1-26): sequential accumulation
// acc = fma(A[y,p], B[p,x], acc) for p = 0..k-1, then the epilogue
// `acc *= alpha; acc += c * beta` evaluated the way nvcc contracts it in the
// reference (basic.cuh:21-24): C = fma(acc, alpha, c * beta).  Outputs equal
// the reference kernel's bit for bit.  Like the reference it always reads C.
//
// Also here: the bounded-wait self-test (sgemm_b200_selftest_wait_timeout).
#include <algorithm>

#include "common.h"
#include "ptx.cuh"
#include "rng.h"

namespace sgb {

__global__ void basic_kernel(int m, int n, int k, float alpha, const float* __restrict__ A, int lda,
                             const float* __restrict__ B, int ldb, float beta, float* C, int ldc) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= n || y >= m) return;
    float acc = 0.0f;
    for (int p = 0; p < k; ++p) acc = fmaf(A[(int64_t)y * lda + p], B[(int64_t)p * ldb + x], acc);
    const float c = C[(int64_t)y * ldc + x];
    C[(int64_t)y * ldc + x] = fmaf(acc, alpha, __fmul_rn(c, beta));
}

// Element (r, c) gets rng_value(key, r * cols + c): the value depends only on
// the seed, the tag and that flat index, whatever the row pitch.  Blocks
// stride over rows along the grid's y, each thread makes 4 consecutive
// columns per step, and when rows start 16-byte aligned (vec) a step is one
// float4 store; no 64-bit division per element.  The two 64-bit multiplies of
// the mixing function per element then bound it (integer throughput), not
// the stores.
__global__ void fill_kernel(float* X, int rows, int cols, int ld, uint64_t seed, uint32_t tag,
                            int dist, int vec) {
    const uint64_t key = rng_key(seed, tag);
    for (int r = blockIdx.y; r < rows; r += gridDim.y) {
        float* row = X + (int64_t)r * ld;
        const uint64_t base = (uint64_t)r * (uint64_t)cols;
        for (int c = 4 * (blockIdx.x * blockDim.x + threadIdx.x); c < cols;
             c += 4 * gridDim.x * blockDim.x) {
            float v[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) v[e] = rng_value(key, base + (uint64_t)(c + e), dist);
            if (vec && c + 3 < cols) {
                *reinterpret_cast<float4*>(row + c) = make_float4(v[0], v[1], v[2], v[3]);
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    if (c + e < cols) row[c + e] = v[e];
            }
        }
    }
}

// The failure path every TMA/MMA wait in the GEMM kernels takes, run on
// purpose: one thread waits, bounded by limit_ns of wall time, for an mbarrier
// phase that nothing will ever complete (no copy and no arrival is issued),
// then records SGEMM_B200_ERR_TIMEOUT in the status word as the GEMM kernels
// do, and returns.  Nothing faults and nothing hangs; the context stays usable.
__global__ void wait_selftest_kernel(int* status, uint64_t limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    fence_barrier_init();
    if (!mbar_wait_for(&bar, 0, limit_ns)) atomicExch(status, SGEMM_B200_ERR_TIMEOUT);
}

}  // namespace sgb

extern "C" int sgemm_b200_selftest_wait_timeout(int limit_us, sgemm_b200_stream_t stream) {
    if (limit_us <= 0 || limit_us > 10000000) {
        sgb::set_last_status(SGEMM_B200_ERR_INVALID_ARG);
        return SGEMM_B200_ERR_INVALID_ARG;
    }
    int s = SGEMM_B200_OK;
    int* status = sgb::device_status_ptr();
    if (!sgb::device_is_sm100())
        s = SGEMM_B200_ERR_UNSUPPORTED;
    else if (!status)
        s = SGEMM_B200_ERR_CUDA;
    else {
        sgb::wait_selftest_kernel<<<1, 32, 0, sgb::as_stream(stream)>>>(
            status, static_cast<uint64_t>(limit_us) * 1000ull);
        s = sgb::cuda_status(cudaGetLastError());
    }
    sgb::set_last_status(s);
    return s;
}

extern "C" int sgemm_b200_basic(int m, int n, int k, const float* alpha, const float* A, int lda,
                                const float* B, int ldb, const float* beta, float* C, int ldc,
                                sgemm_b200_stream_t stream) {
    int s = sgb::check_gemm_args(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    if (s == SGEMM_B200_OK && m > 0 && n > 0) {
        dim3 block(16, 16);
        dim3 grid(sgb::div_up(n, 16), sgb::div_up(m, 16));
        sgb::basic_kernel<<<grid, block, 0, sgb::as_stream(stream)>>>(m, n, k, *alpha, A, lda, B,
                                                                      ldb, *beta, C, ldc);
        s = sgb::cuda_status(cudaGetLastError());
    }
    sgb::set_last_status(s);
    return s;
}

extern "C" void sgemm_basic(int m, int n, int k, const float* alpha, float* A, int lda, float* B,
                            int ldb, const float* beta, float* C, int ldc) {
    sgemm_b200_basic(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, nullptr);
}

extern "C" int sgemm_b200_fill_random(float* X, int rows, int cols, int ld, uint64_t seed,
                                      uint32_t tag, int dist, sgemm_b200_stream_t stream) {
    if (rows < 0 || cols < 0 || ld < cols || dist < 0 || dist > 2) {
        sgb::set_last_status(SGEMM_B200_ERR_INVALID_ARG);
        return SGEMM_B200_ERR_INVALID_ARG;
    }
    if (rows == 0 || cols == 0) return SGEMM_B200_OK;
    if (!X) return SGEMM_B200_ERR_INVALID_ARG;
    const int threads = 256;
    const int vec = (ld % 4 == 0) && (reinterpret_cast<uintptr_t>(X) % 16 == 0);
    // about 16 blocks per SM in all, each striding over rows: long-lived
    // blocks instead of one short block per 1024-column row slab
    const int gx = std::min((cols + 4 * threads - 1) / (4 * threads), 1024);
    const int sms = sgb::device_info().sm_count > 0 ? sgb::device_info().sm_count : 148;
    const int gy = std::min({rows, 65535, std::max(1, (sms * 16 + gx - 1) / gx)});
    const dim3 grid(gx, gy);
    sgb::fill_kernel<<<grid, threads, 0, sgb::as_stream(stream)>>>(X, rows, cols, ld, seed, tag,
                                                                   dist, vec);
    int s = sgb::cuda_status(cudaGetLastError());
    sgb::set_last_status(s);
    return s;
}
