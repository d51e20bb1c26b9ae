// ref_sgemm.cu — TEST INFRASTRUCTURE ONLY.  Exposes the reference's own
// sgemm() and sgemm_basic() (szrlee/sgemm.cu, src/sgemm.cuh:19-113) under C
// linkage so the parity tests and the benchmark's reference arm can call the
// unmodified reference kernels.  The reference sources are NOT copied here:
// oracle/Makefile compiles this file with -I pointing at the reference's
// src/ and common/ directories and -DGPUCC=100, writing oracle/_ref/.
//
// The reference header defines sgemm()/sgemm_basic() non-inline, so it is
// included in exactly this one translation unit (as test.cu:3 does).
#include <sgemm.cuh>

extern "C" void ref_sgemm(int m, int n, int k, const float* alpha, float* A, int lda, float* B,
                          int ldb, const float* beta, float* C, int ldc) {
    sgemm(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

extern "C" void ref_sgemm_basic(int m, int n, int k, const float* alpha, float* A, int lda,
                                float* B, int ldb, const float* beta, float* C, int ldc) {
    sgemm_basic(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

// Which reference kernel sgemm() launches for this shape (src/sgemm.cuh:41-48):
// 1 = sgemm_128x256x8, 0 = sgemm_128x128x8.
extern "C" int ref_sgemm_kernel_choice(int m, int n) { return (m > 2500 || n > 2500) ? 1 : 0; }
