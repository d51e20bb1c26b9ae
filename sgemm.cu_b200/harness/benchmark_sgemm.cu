// benchmark_sgemm.cu — GFLOP/s sweep through the public API, the reference's
// benchmark lane (benchmark.cu:22-208, benchmark.sh:1-43) rebuilt on this
// library.
//
// Protocol kept from the reference: a warm-up of wniter calls at wmsize^3;
// then sizes mmin + i*mstep for i < npts, each with
// n_iter = max(1000*exp(-(s - mmin)/3100), 4) iterations (benchmark.cu:141) of
// event record -> GEMM -> event record -> sync -> L2 flush; GFLOP/s from the
// mean of the second half of the iterations (benchmark.cu:176-183), written as
// `matsize gflops` lines to savedir/fname.txt (benchmark.cu:199-206), which
// the reference's plot script reads unchanged.  Additions: p50/p99 of the
// per-iteration times on stdout, --path (plain|bf16x6|tf32x3), --alpha/--beta,
// --dist, and the L2 flush buffer is allocated once (the reference mallocs it
// on every iteration, common/helper_cuda.h:70-83).
//
// --lib=cublas times cublasSgemm instead (the reference's -DCUBLAS=1 lane,
// benchmark.cu:150-164): row-major C = A*B issued as the column-major
// C^T = B^T * A^T, default math mode (no TF32).
#include <cublas_v2.h>

#include <algorithm>
#include <filesystem>
#include <fstream>

#include "harness_common.h"

int main(int argc, char** argv) {
    using namespace harness;
    const int wniter = flag_int(argc, argv, "wniter", 10);
    const int wmsize = flag_int(argc, argv, "wmsize", 1024);
    const int mmin = flag_int(argc, argv, "mmin", 1024);
    const int mstep = flag_int(argc, argv, "mstep", 128);
    const int npts = flag_int(argc, argv, "npts", 10);
    const std::string fname = flag_str(argc, argv, "fname", "sgemm_b200");
    const std::string savedir = flag_str(argc, argv, "savedir", "benchmark_results");
    const int path = parse_path(flag_str(argc, argv, "path", "plain"));
    const int dist = parse_dist(flag_str(argc, argv, "dist", "u01"));
    const float alpha = (float)flag_double(argc, argv, "alpha", 1.0);
    const float beta = (float)flag_double(argc, argv, "beta", 0.0);
    const bool use_cublas = flag_str(argc, argv, "lib", "sgemm_b200") == "cublas";
    cublasHandle_t handle = nullptr;
    if (use_cublas && cublasCreate(&handle) != CUBLAS_STATUS_SUCCESS) {
        std::fprintf(stderr, "cublasCreate failed\n");
        return 2;
    }
    auto gemm = [&](int s, float* A, float* B, float* C) {
        if (use_cublas) {
            if (cublasSgemm(handle, CUBLAS_OP_N, CUBLAS_OP_N, s, s, s, &alpha, B, s, A, s, &beta,
                            C, s) != CUBLAS_STATUS_SUCCESS) {
                std::fprintf(stderr, "cublasSgemm failed\n");
                std::exit(2);
            }
        } else {
            SCHECK(sgemm_b200_gemm(path, s, s, s, &alpha, A, s, B, s, &beta, C, s, nullptr));
        }
    };

    int dev = 0, l2 = 0;
    HCHECK(cudaGetDevice(&dev));
    HCHECK(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
    void* flush = nullptr;
    const size_t flush_bytes = (size_t)l2 * 2;
    HCHECK(cudaMalloc(&flush, flush_bytes));

    // Warm-up (benchmark.cu:75-97).
    {
        const int s = wmsize;
        float *A, *B, *C;
        HCHECK(cudaMalloc(&A, sizeof(float) * (size_t)s * s));
        HCHECK(cudaMalloc(&B, sizeof(float) * (size_t)s * s));
        HCHECK(cudaMalloc(&C, sizeof(float) * (size_t)s * s));
        SCHECK(sgemm_b200_fill_random(A, s, s, s, 7, 1, dist, nullptr));
        SCHECK(sgemm_b200_fill_random(B, s, s, s, 7, 2, dist, nullptr));
        SCHECK(sgemm_b200_fill_random(C, s, s, s, 7, 3, dist, nullptr));
        for (int i = 0; i < wniter; ++i) {
            gemm(s, A, B, C);
            HCHECK(cudaDeviceSynchronize());
        }
        HCHECK(cudaFree(A));
        HCHECK(cudaFree(B));
        HCHECK(cudaFree(C));
    }

    std::vector<int> sizes, gflops;
    for (int i = 0; i < npts; ++i) {
        const int s = mmin + i * mstep;
        float *A, *B, *C;
        HCHECK(cudaMalloc(&A, sizeof(float) * (size_t)s * s));
        HCHECK(cudaMalloc(&B, sizeof(float) * (size_t)s * s));
        HCHECK(cudaMalloc(&C, sizeof(float) * (size_t)s * s));
        SCHECK(sgemm_b200_fill_random(A, s, s, s, 11, 1, dist, nullptr));
        SCHECK(sgemm_b200_fill_random(B, s, s, s, 11, 2, dist, nullptr));
        SCHECK(sgemm_b200_fill_random(C, s, s, s, 11, 3, dist, nullptr));
        const double gflop = 2.0 * s * (double)s * s * 1e-9;
        const int n_iter = std::max((int)(1000 * std::exp((-s + mmin) / 3100.0)), 4);
        std::vector<float> ms(n_iter);
        cudaEvent_t e0, e1;
        HCHECK(cudaEventCreate(&e0));
        HCHECK(cudaEventCreate(&e1));
        for (int j = 0; j < n_iter; ++j) {
            HCHECK(cudaEventRecord(e0));
            gemm(s, A, B, C);
            HCHECK(cudaEventRecord(e1));
            HCHECK(cudaEventSynchronize(e1));
            HCHECK(cudaEventElapsedTime(&ms[j], e0, e1));
            HCHECK(cudaMemsetAsync(flush, j & 0xff, flush_bytes));
        }
        double avg = 0;
        const int mid = n_iter / 2;
        for (int j = mid; j < n_iter; ++j) avg += ms[j];
        avg /= (n_iter - mid);
        std::vector<float> sorted(ms.begin() + mid, ms.end());
        std::sort(sorted.begin(), sorted.end());
        const float p50 = sorted[sorted.size() / 2];
        const float p99 = sorted[std::min(sorted.size() - 1, (size_t)(0.99 * sorted.size()))];
        const int g = (int)(gflop / (avg * 1e-3));
        sizes.push_back(s);
        gflops.push_back(g);
        std::printf("m=n=k=%i:\n%s %8i GFLOP/s  (p50 %.3f ms, p99 %.3f ms)\n\n", s, fname.c_str(),
                    g, p50, p99);
        HCHECK(cudaEventDestroy(e0));
        HCHECK(cudaEventDestroy(e1));
        HCHECK(cudaFree(A));
        HCHECK(cudaFree(B));
        HCHECK(cudaFree(C));
    }
    std::filesystem::create_directories(savedir);
    const std::string out = savedir + "/" + fname + ".txt";
    std::ofstream f(out);
    for (size_t i = 0; i < sizes.size(); ++i) f << sizes[i] << " " << gflops[i] << "\n";
    std::printf("Benchmark data stored in %s\n", out.c_str());
    HCHECK(cudaFree(flush));
    if (handle) cublasDestroy(handle);
    return 0;
}
