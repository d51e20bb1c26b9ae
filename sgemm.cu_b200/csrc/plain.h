// plain.h — internal interface of the plain FFMA path (used by the grouped
// kernel's sequential baseline, the autotuner and the serving loop).
#pragma once

#include <cuda_runtime.h>

namespace sgb {

int plain_config_count();
const char* plain_config_name(int cfg);
int plain_config_tile(int cfg, int* bm, int* bn);
int plain_select(int m, int n, int k, const float* A, int lda, const float* B, int ldb,
                 bool reads_c);
int plain_launch(int cfg, int m, int n, int k, float alpha, const float* A, int lda,
                 const float* B, int ldb, float beta, float* C, int ldc, cudaStream_t stream);
// The same GEMM over one k range of a longer product whose accumulators are
// carried between launches in an m x n row-major buffer (pitch ld_acc, 16-byte
// aligned): acc_in (or null: start from zero) seeds them, acc_out (or null:
// apply alpha/beta and write C) receives the unscaled sums.  k ranges that
// start on multiples of 32 give the one-launch product's bits.
int plain_launch_acc(int cfg, int m, int n, int k, float alpha, const float* A, int lda,
                     const float* B, int ldb, float beta, float* C, int ldc, const float* acc_in,
                     float* acc_out, int ld_acc, cudaStream_t stream);

}  // namespace sgb
