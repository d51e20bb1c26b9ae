// oracle_gpu.cu — TEST INFRASTRUCTURE ONLY.  FP64 GEMM on the GPU used as the
// accuracy oracle at sizes the CPU FP64 GEMM (oracle.c) cannot finish quickly
// (8192^3, 16384^3).  Never linked into or called by the product library; the
// tests cross-check it against oracle.c's oracle_dgemm_rows on sampled rows.
//
//   REF = alpha * A * B + beta * C0           (FP64 products and sums)
//   MAG = |alpha| * |A||B| + |beta| * |C0|    (for the componentwise error)
//
// Plain tiled SIMT FP64 kernel: 64x64 tile, 16-deep k step, 256 threads with
// 4x4 outputs each.  Correctness over speed.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace {

constexpr int T = 64, KT = 16;

__global__ void dgemm_kernel(int m, int n, int k, double alpha, const float* __restrict__ A,
                             int lda, const float* __restrict__ B, int ldb, double beta,
                             const float* __restrict__ C0, int ldc0, double* __restrict__ REF,
                             double* __restrict__ MAG) {
    __shared__ double As[KT][T + 1];
    __shared__ double Bs[KT][T + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int m0 = blockIdx.y * T, n0 = blockIdx.x * T;
    double acc[4][4] = {}, mag[4][4] = {};
    for (int k0 = 0; k0 < k; k0 += KT) {
        for (int e = threadIdx.x; e < T * KT; e += 256) {
            const int r = e / KT, c = e % KT;  // A tile: row r, k c
            const int gr = m0 + r, gk = k0 + c;
            As[c][r] = (gr < m && gk < k) ? (double)A[(int64_t)gr * lda + gk] : 0.0;
            const int br = e / T, bc = e % T;  // B tile: k br, col bc
            const int gbk = k0 + br, gbc = n0 + bc;
            Bs[br][bc] = (gbk < k && gbc < n) ? (double)B[(int64_t)gbk * ldb + gbc] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KT; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    acc[i][j] = fma(a[i], b[j], acc[i][j]);
                    mag[i][j] = fma(fabs(a[i]), fabs(b[j]), mag[i][j]);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = m0 + ty + 16 * i;
        if (r >= m) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = n0 + tx + 16 * j;
            if (c >= n) continue;
            const double c0 = (C0 && beta != 0.0) ? (double)C0[(int64_t)r * ldc0 + c] : 0.0;
            REF[(int64_t)r * n + c] = alpha * acc[i][j] + beta * c0;
            if (MAG) MAG[(int64_t)r * n + c] = fabs(alpha) * mag[i][j] + fabs(beta) * fabs(c0);
        }
    }
}

__global__ void maxabs_kernel(int64_t count, const double* __restrict__ ref, double* partial) {
    __shared__ double red[256];
    double mx = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x)
        mx = fmax(mx, fabs(ref[i]));
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// Per block: [max rel, sum rel, count rel, max componentwise, non-finite count]
__global__ void stats_kernel(int64_t count, int n, const float* __restrict__ C, int ldc,
                             const double* __restrict__ ref, const double* __restrict__ mag,
                             double thresh, double* partial) {
    __shared__ double r0[256], r1[256], r2[256], r3[256], r4[256];
    double mx = 0, sum = 0, cnt = 0, cw = 0, bad = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / n, c = i % n;
        const double v = C[r * ldc + c];
        if (!isfinite(v)) {
            bad += 1;
            continue;
        }
        const double d = fabs(v - ref[i]);
        const double a = fabs(ref[i]);
        if (a >= thresh && a != 0.0) {
            const double e = d / a;
            mx = fmax(mx, e);
            sum += e;
            cnt += 1;
        }
        if (mag && mag[i] > 0.0) cw = fmax(cw, d / mag[i]);
    }
    r0[threadIdx.x] = mx;
    r1[threadIdx.x] = sum;
    r2[threadIdx.x] = cnt;
    r3[threadIdx.x] = cw;
    r4[threadIdx.x] = bad;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            r0[threadIdx.x] = fmax(r0[threadIdx.x], r0[threadIdx.x + s]);
            r1[threadIdx.x] += r1[threadIdx.x + s];
            r2[threadIdx.x] += r2[threadIdx.x + s];
            r3[threadIdx.x] = fmax(r3[threadIdx.x], r3[threadIdx.x + s]);
            r4[threadIdx.x] += r4[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double* o = partial + 5 * blockIdx.x;
        o[0] = r0[0];
        o[1] = r1[0];
        o[2] = r2[0];
        o[3] = r3[0];
        o[4] = r4[0];
    }
}

}  // namespace

extern "C" int oracle_gpu_dgemm(int m, int n, int k, double alpha, const float* A, int lda,
                                const float* B, int ldb, double beta, const float* C0, int ldc0,
                                double* REF, double* MAG) {
    if (m <= 0 || n <= 0) return 0;
    dim3 grid((n + T - 1) / T, (m + T - 1) / T);
    dgemm_kernel<<<grid, 256>>>(m, n, k, alpha, A, lda, B, ldb, beta, C0, ldc0, REF, MAG);
    if (cudaGetLastError() != cudaSuccess) return 1;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

// out: [max rel, mean rel, max componentwise, count rel, non-finite]
extern "C" int oracle_gpu_error_stats(int m, int n, const float* C, int ldc, const double* REF,
                                      const double* MAG, double* out) {
    const int64_t count = (int64_t)m * n;
    const int blocks = 1024;
    double* part = nullptr;
    if (cudaMalloc(&part, sizeof(double) * 5 * blocks) != cudaSuccess) return 1;
    double host[5 * 1024];
    maxabs_kernel<<<blocks, 256>>>(count, REF, part);
    if (cudaMemcpy(host, part, sizeof(double) * blocks, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaFree(part);
        return 1;
    }
    double mx = 0;
    for (int i = 0; i < blocks; ++i) mx = fmax(mx, host[i]);
    stats_kernel<<<blocks, 256>>>(count, n, C, ldc, REF, MAG, 1e-3 * mx, part);
    if (cudaMemcpy(host, part, sizeof(double) * 5 * blocks, cudaMemcpyDeviceToHost) !=
        cudaSuccess) {
        cudaFree(part);
        return 1;
    }
    cudaFree(part);
    double mrel = 0, sum = 0, cnt = 0, cw = 0, bad = 0;
    for (int i = 0; i < blocks; ++i) {
        mrel = fmax(mrel, host[5 * i]);
        sum += host[5 * i + 1];
        cnt += host[5 * i + 2];
        cw = fmax(cw, host[5 * i + 3]);
        bad += host[5 * i + 4];
    }
    out[0] = mrel;
    out[1] = cnt > 0 ? sum / cnt : 0.0;
    out[2] = cw;
    out[3] = cnt;
    out[4] = bad;
    return 0;
}
