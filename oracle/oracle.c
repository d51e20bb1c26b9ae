/*
 * oracle.c — TEST INFRASTRUCTURE ONLY.  CPU restatement of the reference's
 * correctness oracle and the FP64 checker.  Nothing in the product library
 * links, loads or calls this file; only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg do, as the checker.
 *
 * Contents
 *  - oracle_fill: seeded counter-based generator (restates the generator the
 *    library's fill kernel uses; see rng_* below).
 *  - oracle_sgemm_basic: the reference's per-element arithmetic, in two
 *    epilogue flavours (the accumulation is the same for both):
 *        acc = 0; for p in 0..k-1: acc = fma(A[y,p], B[p,x], acc)
 *    (kernel_basic, src/kernels/basic.cuh:18-20; the tiled kernels'
 *    increasing-k chain, src/kernels/128x256x8.cuh:224-239), then
 *      basic == 0, the tiled kernels (128x256x8.cuh:331-337, :365-380):
 *        v = acc * alpha;  C = beta != 0 ? fma(C, beta, v) : v   (C unread)
 *      basic == 1, kernel_basic (basic.cuh:21-24), as nvcc contracts
 *        `acc *= alpha; acc += c * beta` (default --fmad=true):
 *        C = fma(acc, alpha, C * beta)                          (C always read)
 *    Both flavours are pinned bit-for-bit to the reference's own outputs
 *    (tests/golden/).  The per-element summation order is kept (i-p-j loop,
 *    j vectorised), so results equal the naive order's bit for bit.
 *  - oracle_dgemm / oracle_dgemm_rows: FP64 C64 = alpha*A*B + beta*C0 with
 *    exact products (24-bit x 24-bit fits in 53 bits) and FP64 sums, plus the
 *    magnitude |alpha|*(|A||B|) + |beta|*|C0| used by the componentwise error.
 *  - oracle_error_stats: max/mean relative error over elements with
 *    |c64| >= 1e-3 * max|c64|, and max componentwise error.
 *
 * Parity pins: tests/golden/ holds outputs of the reference's own kernels
 * (sgemm() and sgemm_basic() built from the reference sources for sm_100a)
 * generated by tests/golden/make_golden.py; tests/test_oracle.py checks this
 * file reproduces them.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------- generator -- */

/* SplitMix64 finaliser (Steele, Lea, Flood, OOPSLA 2014). */
static inline uint64_t rng_mix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline uint64_t rng_key(uint64_t seed, uint32_t tag) {
    return rng_mix(seed ^ rng_mix(0xA0761D6478BD642Full + (uint64_t)tag));
}

static inline float rng_value(uint64_t key, uint64_t index, int dist) {
    uint64_t b = rng_mix(key + index);
    if (dist == 0) {
        int32_t u = (int32_t)(b >> 40) - (1 << 23);
        return (float)u * (1.0f / 8388608.0f);
    }
    if (dist == 1) return (float)(uint32_t)(b >> 40) * (1.0f / 16777216.0f);
    uint32_t sign = (uint32_t)(b & 1u) << 31;
    int32_t e = (int32_t)((b >> 1) % 21u) - 10;
    uint32_t mant = (uint32_t)(b >> 41) & 0x7FFFFFu;
    uint32_t bits = sign | ((uint32_t)(127 + e) << 23) | mant;
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

int oracle_fill(float* X, int rows, int cols, int ld, uint64_t seed, uint32_t tag, int dist) {
    if (rows < 0 || cols < 0 || ld < cols || dist < 0 || dist > 2) return 1;
    const uint64_t key = rng_key(seed, tag);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c)
            X[(int64_t)r * ld + c] = rng_value(key, (uint64_t)r * cols + c, dist);
    return 0;
}

/* Fill only the listed rows of a rows x cols matrix (row r of the full matrix
 * goes to out[i * cols], i = position of r in the list). */
int oracle_fill_rows(float* out, const int* row_ids, int nrows, int cols, uint64_t seed,
                     uint32_t tag, int dist) {
    const uint64_t key = rng_key(seed, tag);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nrows; ++i)
        for (int c = 0; c < cols; ++c)
            out[(int64_t)i * cols + c] = rng_value(key, (uint64_t)row_ids[i] * cols + c, dist);
    return 0;
}

/* --------------------------------------------------- FP32 FMA-chain GEMM -- */

#define IB 8   /* rows per block: their accumulators stay in L1 together */
#define JB 256 /* columns per block */

#if defined(__x86_64__)
#define FMA_TARGET __attribute__((target("avx2,fma")))
#else
#define FMA_TARGET
#endif

/* One IB x JB block of C rows [i0, i0+ib) x cols [j0, j0+jb); rows of A are
 * given by a_rows[i] (row pointers) so row subsets work too. */
#define BLOCK_BODY                                                                   \
    float acc[IB][JB];                                                               \
    for (int i = 0; i < ib; ++i)                                                     \
        for (int j = 0; j < jb; ++j) acc[i][j] = 0.0f;                               \
    for (int p = 0; p < k; ++p) {                                                    \
        const float* brow = B + (int64_t)p * ldb + j0;                               \
        for (int i = 0; i < ib; ++i) {                                               \
            const float a = a_rows[i][p];                                            \
            for (int j = 0; j < jb; ++j) acc[i][j] = fmaf(a, brow[j], acc[i][j]);    \
        }                                                                            \
    }                                                                                \
    for (int i = 0; i < ib; ++i) {                                                   \
        float* crow = c_rows[i] + j0;                                                \
        for (int j = 0; j < jb; ++j) {                                               \
            float v;                                                                 \
            if (basic) {                                                             \
                const float cb = crow[j] * beta;                                     \
                v = fmaf(acc[i][j], alpha, cb);                                      \
            } else {                                                                 \
                v = acc[i][j] * alpha;                                               \
                if (beta != 0.0f) v = fmaf(crow[j], beta, v);                        \
            }                                                                        \
            crow[j] = v;                                                             \
        }                                                                            \
    }

FMA_TARGET static void block_fma(int ib, int jb, int j0, int k, float alpha,
                                 const float* const* a_rows, const float* B, int ldb, float beta,
                                 float* const* c_rows, int basic) {
    BLOCK_BODY
}

static void block_plain(int ib, int jb, int j0, int k, float alpha, const float* const* a_rows,
                        const float* B, int ldb, float beta, float* const* c_rows,
                        int basic) {
    BLOCK_BODY
}

static int have_fma(void) {
#if defined(__x86_64__)
    return __builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma");
#else
    return 0;
#endif
}

static void set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* C rows listed in row_ids (C_rows[i] is the output row for A row row_ids[i]):
 * the general form behind both entry points below. */
static int sgemm_rows_impl(int nrows, const int* row_ids, int n, int k, float alpha,
                           const float* A, int lda, const float* B, int ldb, float beta,
                           float* C, int ldc, int c_is_compact, int basic,
                           int nthreads) {
    if (nrows < 0 || n < 0 || k < 0) return 1;
    set_threads(nthreads);
    const int fma_ok = have_fma();
    const int nblk = (nrows + IB - 1) / IB;
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nblk; ++b) {
        const int i0 = b * IB;
        const int ib = nrows - i0 < IB ? nrows - i0 : IB;
        const float* a_rows[IB];
        float* c_rows[IB];
        for (int i = 0; i < ib; ++i) {
            const int r = row_ids ? row_ids[i0 + i] : i0 + i;
            a_rows[i] = A + (int64_t)r * lda;
            c_rows[i] = C + (int64_t)(c_is_compact ? i0 + i : r) * ldc;
        }
        for (int j0 = 0; j0 < n; j0 += JB) {
            const int jb = n - j0 < JB ? n - j0 : JB;
            if (fma_ok)
                block_fma(ib, jb, j0, k, alpha, a_rows, B, ldb, beta, c_rows, basic);
            else
                block_plain(ib, jb, j0, k, alpha, a_rows, B, ldb, beta, c_rows,
                            basic);
        }
    }
    return 0;
}

int oracle_sgemm_basic(int m, int n, int k, float alpha, const float* A, int lda, const float* B,
                       int ldb, float beta, float* C, int ldc, int basic,
                       int nthreads) {
    return sgemm_rows_impl(m, NULL, n, k, alpha, A, lda, B, ldb, beta, C, ldc, 0,
                           basic, nthreads);
}

/* Rows row_ids[0..nrows) of the product; A is the full matrix, C is compact
 * (nrows x n, row stride ldc) and holds the beta-input rows on entry. */
int oracle_sgemm_basic_rows(int nrows, const int* row_ids, int n, int k, float alpha,
                            const float* A, int lda, const float* B, int ldb, float beta,
                            float* C, int ldc, int basic, int nthreads) {
    return sgemm_rows_impl(nrows, row_ids, n, k, alpha, A, lda, B, ldb, beta, C, ldc, 1,
                           basic, nthreads);
}

/* ------------------------------------------------------------ FP64 GEMM -- */

/* C64[i,:] = alpha * sum_p A[r_i,p] * B[p,:] + beta * C0[i,:]  and
 * MAG[i,:] = |alpha| * sum_p |A[r_i,p]| |B[p,:]| + |beta| |C0[i,:]|
 * for the listed rows (all rows if row_ids is NULL).  C0 is compact (nrows x
 * n, stride ldc0) or NULL when beta == 0.  Outputs are compact nrows x n. */
int oracle_dgemm_rows(int nrows, const int* row_ids, int n, int k, double alpha, const float* A,
                      int lda, const float* B, int ldb, double beta, const float* C0, int ldc0,
                      double* C64, double* MAG, int nthreads) {
    if (nrows < 0 || n < 0 || k < 0) return 1;
    set_threads(nthreads);
    const int nblk = (nrows + IB - 1) / IB;
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nblk; ++b) {
        const int i0 = b * IB;
        const int ib = nrows - i0 < IB ? nrows - i0 : IB;
        double acc[IB][JB], mag[IB][JB];
        for (int j0 = 0; j0 < n; j0 += JB) {
            const int jb = n - j0 < JB ? n - j0 : JB;
            for (int i = 0; i < ib; ++i)
                for (int j = 0; j < jb; ++j) acc[i][j] = mag[i][j] = 0.0;
            for (int p = 0; p < k; ++p) {
                const float* brow = B + (int64_t)p * ldb + j0;
                for (int i = 0; i < ib; ++i) {
                    const int r = row_ids ? row_ids[i0 + i] : i0 + i;
                    const double a = A[(int64_t)r * lda + p];
                    const double aa = fabs(a);
                    for (int j = 0; j < jb; ++j) {
                        const double bb = brow[j];
                        acc[i][j] += a * bb;
                        mag[i][j] += aa * fabs(bb);
                    }
                }
            }
            for (int i = 0; i < ib; ++i)
                for (int j = 0; j < jb; ++j) {
                    double c0 = 0.0;
                    if (C0 && beta != 0.0) c0 = C0[(int64_t)(i0 + i) * ldc0 + j0 + j];
                    C64[(int64_t)(i0 + i) * n + j0 + j] = alpha * acc[i][j] + beta * c0;
                    if (MAG)
                        MAG[(int64_t)(i0 + i) * n + j0 + j] =
                            fabs(alpha) * mag[i][j] + fabs(beta) * fabs(c0);
                }
        }
    }
    return 0;
}

/* ----------------------------------------------------------- error stats -- */

/* out[0] = max rel err over |ref| >= 1e-3 max|ref|; out[1] = mean of the same;
 * out[2] = max componentwise err |c-ref| / mag; out[3] = count of elements in
 * the relative set; out[4] = number of non-finite results. */
int oracle_error_stats(int64_t count, const float* C, const double* ref, const double* mag,
                       double* out) {
    double maxabs = 0.0;
    for (int64_t i = 0; i < count; ++i) {
        const double a = fabs(ref[i]);
        if (a > maxabs) maxabs = a;
    }
    const double thresh = 1e-3 * maxabs;
    double mx = 0.0, sum = 0.0, cw = 0.0;
    int64_t n = 0, bad = 0;
    for (int64_t i = 0; i < count; ++i) {
        const double c = C[i];
        if (!isfinite(c)) {
            ++bad;
            continue;
        }
        const double d = fabs(c - ref[i]);
        if (fabs(ref[i]) >= thresh && ref[i] != 0.0) {
            const double r = d / fabs(ref[i]);
            if (r > mx) mx = r;
            sum += r;
            ++n;
        }
        if (mag && mag[i] > 0.0) {
            const double e = d / mag[i];
            if (e > cw) cw = e;
        }
    }
    out[0] = mx;
    out[1] = n ? sum / (double)n : 0.0;
    out[2] = cw;
    out[3] = (double)n;
    out[4] = (double)bad;
    return 0;
}
