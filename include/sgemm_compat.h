/*
 * sgemm_compat.h — drop-in for the reference's launch surface.
 *
 * A translation unit that did `#include <sgemm.cuh>` (szrlee/sgemm.cu) can
 * include this header instead and link libsgemm_b200.so.  The two functions
 * keep the reference's exact parameter lists:
 *
 *   sgemm()        replaces src/sgemm.cuh:19-90
 *   sgemm_basic()  replaces src/sgemm.cuh:92-113
 *
 * Both run on the legacy default stream and return without synchronising,
 * like the reference.  They return void, as the reference does; the status of
 * the last call is available from sgemm_b200_last_status().  A and B are
 * non-const in the signature (as in the reference) but are never written.
 *
 * Differences from the reference, all in the caller's favour:
 *  - general ldb and ldc are honoured (the reference needs ldb == ldc == n);
 *  - the function is declared here and defined once in the library, so any
 *    number of translation units may include this header (the reference
 *    defines sgemm() non-inline in its header, so only one may).
 */
#ifndef SGEMM_COMPAT_H
#define SGEMM_COMPAT_H

#include "sgemm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

void sgemm(int m, int n, int k,
           const float* alpha,
           float* A, int lda,
           float* B, int ldb,
           const float* beta,
           float* C, int ldc);

void sgemm_basic(int m, int n, int k,
                 const float* alpha,
                 float* A, int lda,
                 float* B, int ldb,
                 const float* beta,
                 float* C, int ldc);

#ifdef __cplusplus
}
#endif

#endif /* SGEMM_COMPAT_H */
