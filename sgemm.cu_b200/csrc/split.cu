// split.cu — split-precision tensor-core path (under construction).
#include "common.h"

extern "C" size_t sgemm_b200_split_workspace_size(int path, int m, int n, int k) {
    (void)path; (void)m; (void)n; (void)k;
    return 0;
}

extern "C" int sgemm_b200_split(int path, int m, int n, int k, const float* alpha, const float* A,
                                int lda, const float* B, int ldb, const float* beta, float* C,
                                int ldc, void* workspace, size_t workspace_bytes,
                                sgemm_b200_stream_t stream) {
    (void)path; (void)m; (void)n; (void)k; (void)alpha; (void)A; (void)lda; (void)B; (void)ldb;
    (void)beta; (void)C; (void)ldc; (void)workspace; (void)workspace_bytes; (void)stream;
    sgb::set_last_status(SGEMM_B200_ERR_UNSUPPORTED);
    return SGEMM_B200_ERR_UNSUPPORTED;
}

extern "C" int sgemm_b200_gemm(int path, int m, int n, int k, const float* alpha, const float* A,
                               int lda, const float* B, int ldb, const float* beta, float* C,
                               int ldc, sgemm_b200_stream_t stream) {
    if (path == SGEMM_B200_PATH_PLAIN)
        return sgemm_b200(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream);
    return sgemm_b200_split(path, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, nullptr, 0, stream);
}
