/*
 * sgemm_b200.h — C ABI of the B200-native (sm_100a) FP32 GEMM library.
 *
 *   C := alpha * A * B + beta * C        (FP32, row-major, "NN")
 *
 * A is m x k with row stride lda, B is k x n with row stride ldb, C is m x n
 * with row stride ldc, all in elements.  Matrices are caller-owned DEVICE
 * pointers; alpha and beta are caller-owned HOST pointers read by value when
 * the call is made (the reference's convention, src/sgemm.cuh:19-30,44,47).
 * Column-major callers swap (A, lda) and (B, ldb) and exchange m and n,
 * because C^T = B^T * A^T (src/sgemm.cuh:31-33).
 *
 * Every entry point returns an sgemm_b200_status.  Work is enqueued on the
 * given stream and the call returns without synchronising, like the
 * reference's sgemm() (src/sgemm.cuh:35-48), which also never synchronises.
 *
 * Unlike the reference kernels (128x128x8.cuh:263,368 and 128x256x8.cuh:273,
 * 372-380 use n for the B and C row strides), every path here honours general
 * lda >= k, ldb >= n and ldc >= n.  With beta == 0, C is never read, matching
 * the reference's tiled kernels (128x256x8.cuh:365-380).
 */
#ifndef SGEMM_B200_H
#define SGEMM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Version of this C ABI.  It changes whenever an existing entry point changes
 * its parameters or their meaning (new entry points keep it); a caller
 * compiled against one header can compare it with sgemm_b200_abi_version()
 * at run time. */
#define SGEMM_B200_ABI_VERSION 2
int sgemm_b200_abi_version(void);

/* cudaStream_t without pulling in the CUDA headers: the ABI takes it as an
 * opaque pointer (NULL = the legacy default stream). */
typedef void* sgemm_b200_stream_t;

typedef enum {
    SGEMM_B200_OK = 0,
    SGEMM_B200_ERR_INVALID_ARG = 1,   /* negative size, ld too small, NULL pointer */
    SGEMM_B200_ERR_UNSUPPORTED = 2,   /* no sm_100 device, or mode not built */
    SGEMM_B200_ERR_CUDA = 3,          /* a CUDA runtime/driver call failed */
    SGEMM_B200_ERR_TIMEOUT = 4,       /* a bounded device-side wait expired */
    SGEMM_B200_ERR_NO_MEMORY = 5,     /* allocation or workspace too small */
    SGEMM_B200_ERR_REJECTED = 6       /* serving: request refused by admission */
} sgemm_b200_status;

/* Compute paths. */
typedef enum {
    SGEMM_B200_PATH_PLAIN = 0,    /* FFMA on the SIMT pipes, bit-exact with the reference */
    SGEMM_B200_PATH_BF16X6 = 1,   /* 3-way BF16 split, 6 cross products on tcgen05 */
    SGEMM_B200_PATH_TF32X3 = 2    /* 2-way TF32 split, 3 cross products on tcgen05 */
} sgemm_b200_path;

/* ------------------------------------------------------------------------ */
/* Plain FFMA path                                                           */
/* ------------------------------------------------------------------------ */

/* Replaces sgemm() at src/sgemm.cuh:19-48 (the GPUCC >= 80 branch that
 * launches sgemm_128x128x8 / sgemm_128x256x8), adding a stream argument and a
 * status return.  Each C element is accumulated over k in increasing order
 * with one fused multiply-add per term, then acc *= alpha and
 * C = fmaf(C_old, beta, acc), so results equal the reference kernels' bit for
 * bit on the same inputs.  After one call on the device outside stream
 * capture (which caches the device's properties and the library pool), calls
 * can be captured into a CUDA graph, including ones whose unaligned strides
 * take the pack-to-aligned-rows path (its scratch is stream-ordered). */
int sgemm_b200(int m, int n, int k,
               const float* alpha,
               const float* A, int lda,
               const float* B, int ldb,
               const float* beta,
               float* C, int ldc,
               sgemm_b200_stream_t stream);

/* Same computation with an explicit kernel configuration (see
 * sgemm_b200_config_count / sgemm_b200_config_name); cfg < 0 means the
 * dispatcher's choice.  Used by the autotuner and the tests. */
int sgemm_b200_with_config(int cfg, int m, int n, int k,
                           const float* alpha,
                           const float* A, int lda,
                           const float* B, int ldb,
                           const float* beta,
                           float* C, int ldc,
                           sgemm_b200_stream_t stream);

/* Number of compiled plain-path kernel configurations and their names
 * (e.g. "tma_128x64_w4_t8x8_s3"). */
int sgemm_b200_config_count(void);
const char* sgemm_b200_config_name(int cfg);
/* Configuration of the kernel sgemm_b200 runs for this shape and these
 * pointers when C is read (beta != 0); host-only.  C and ldc are not used
 * (kept for callers of the first form of this query).  Strides that TMA
 * cannot describe (not a multiple of 4 floats, or a base not 16-byte aligned)
 * on problems of at least 512^3 are first copied to aligned rows (see
 * sgemm_b200_packs), so the answer is then a TMA configuration; smaller such
 * problems use a cp.async configuration. */
int sgemm_b200_select_config(int m, int n, int k,
                             const float* A, int lda,
                             const float* B, int ldb,
                             const float* C, int ldc);
/* The same query for a given beta (a host pointer, as in sgemm_b200; NULL
 * means C is read): with beta == 0 the dispatcher may pick another tile,
 * because an epilogue that only writes C changes which tile finishes first
 * when the problem is a single partial wave. */
int sgemm_b200_select_config_beta(int m, int n, int k,
                                  const float* A, int lda,
                                  const float* B, int ldb,
                                  const float* beta);

/* Operands sgemm_b200 copies to aligned rows before its kernel (host-only):
 * bit 0 for A, bit 1 for B, 0 when both are read in place.  The copy is one
 * extra kernel launch for both operands. */
int sgemm_b200_packs(int m, int n, int k,
                     const float* A, int lda,
                     const float* B, int ldb);

/* Replaces the reference's pre-Ampere texture path (src/sgemm.cuh:49-89,
 * sgemm_texld_128x128x8 in src/kernels/128x128x8_texld.cuh): when lda and ldb
 * are multiples of 4 and A and B are 16-byte aligned (the reference's
 * is_aligned condition), A and B are read through linear texture objects as
 * float4 texels; otherwise -- and for k == 0, or operands too large for a
 * linear texture -- the call runs sgemm_b200's kernels, as the reference
 * falls back to its plain-load kernel.  Results equal sgemm_b200's bit for
 * bit.  The texture objects are created per call and destroyed once the
 * call's kernel has finished, without the call waiting for it. */
int sgemm_b200_texld(int m, int n, int k,
                     const float* alpha,
                     const float* A, int lda,
                     const float* B, int ldb,
                     const float* beta,
                     float* C, int ldc,
                     sgemm_b200_stream_t stream);

/* Replaces sgemm_basic() at src/sgemm.cuh:92-113 (kernel_basic,
 * src/kernels/basic.cuh:1-26): one thread per C element, sequential
 * accumulation, C always read.  Kept for the reference's test semantics. */
int sgemm_b200_basic(int m, int n, int k,
                     const float* alpha,
                     const float* A, int lda,
                     const float* B, int ldb,
                     const float* beta,
                     float* C, int ldc,
                     sgemm_b200_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Split-precision tensor-core path (no reference counterpart)               */
/* ------------------------------------------------------------------------ */

/* Bytes of device workspace sgemm_b200_split needs for this shape/path. */
size_t sgemm_b200_split_workspace_size(int path, int m, int n, int k);

/* C := alpha*A*B + beta*C with A and B split into BF16 (path BF16X6) or TF32
 * (path TF32X3) terms whose cross products run on tcgen05 with FP32
 * accumulation in tensor memory.  Same argument meaning as sgemm_b200.
 * workspace may be NULL, in which case the call allocates it stream-ordered
 * on `stream` from a memory pool the library keeps per device (freed blocks
 * are reused by later calls). */
int sgemm_b200_split(int path, int m, int n, int k,
                     const float* alpha,
                     const float* A, int lda,
                     const float* B, int ldb,
                     const float* beta,
                     float* C, int ldc,
                     void* workspace, size_t workspace_bytes,
                     sgemm_b200_stream_t stream);

/* Allocation-free split-precision GEMM.  No counterpart in the reference
 * (which never allocates, and has no split path).
 *
 * For callers that must not allocate device memory during a call: code that
 * runs where another component owns the device allocator (a framework that
 * reserved the GPU's memory up front), latency-critical loops in which
 * cudaMalloc/cudaFree would synchronise the device, and fixed-footprint
 * deployments that must not fail for lack of memory at run time.
 *
 * Same arguments and result as sgemm_b200_split, but the split operand planes
 * go to one static device array inside this library instead of a workspace:
 * the call makes no cudaMalloc, cudaFree or other allocation.  The array
 * (64 MiB of planes plus 1 KiB of base alignment) exists on every GPU that
 * loads this library until the process exits.  A problem is accepted when
 * sgemm_b200_split_workspace_size(path, m, n, k) <= 64 MiB + 1 KiB, i.e. its
 * planes fit in 64 MiB: cubes up to m = n = k = 2048 for TF32X3 (planes of
 * exactly 64 MiB) and 2361 for BF16X6; larger problems are refused with
 * SGEMM_B200_ERR_NO_MEMORY before any work is enqueued.  k == 0 (C := beta*C)
 * needs no planes and is always accepted.
 * The first call on each device looks up the array's device address (with
 * that device current); make that first call before any stream capture.
 * Every call shares the one array, so calls whose work overlaps on the GPU
 * (different streams, or different host threads) race: order them on one
 * stream.  Nothing in the array needs clearing between calls; each call
 * rewrites all of the planes it reads. */
int sgemm_b200_split_noalloc(int path, int m, int n, int k,
                             const float* alpha,
                             const float* A, int lda,
                             const float* B, int ldb,
                             const float* beta,
                             float* C, int ldc,
                             sgemm_b200_stream_t stream);

/* Dispatch by path: PLAIN goes to sgemm_b200, the others to sgemm_b200_split
 * with a stream-ordered workspace. */
int sgemm_b200_gemm(int path, int m, int n, int k,
                    const float* alpha,
                    const float* A, int lda,
                    const float* B, int ldb,
                    const float* beta,
                    float* C, int ldc,
                    sgemm_b200_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Host-resident operands (no reference counterpart)                         */
/* ------------------------------------------------------------------------ */

/* C := alpha*A*B + beta*C with A, B and C in HOST memory.  Replaces the
 * reference callers' cudaMemcpy(A,B,C) -> sgemm() -> cudaMemcpy(C) sequence
 * (test.cu:70-80, benchmark.cu:69-73): the library stages the operands in
 * device memory itself, cutting C into blocks (row bands x column chunks,
 * see sgemm_b200_host_plan) so that the host-to-device copies, the block
 * GEMMs (four streams) and the device-to-host copies overlap; large plain
 * problems take the k-outer plan instead (see sgemm_b200_host_plan_kouter).
 * `path` is a sgemm_b200_path; each block is the same GEMM sgemm_b200_gemm()
 * runs, and k slices start on whole 32-deep k blocks, so C is bit-identical
 * to copying everything and calling it once.  Device memory: A, B and C from
 * the library's stream-ordered pool (and, for the k-outer plan, an m x n
 * buffer of FP32 sums).  Stream-ordered on
 * `stream`: C on the host is final once `stream` has synchronised.
 * Page-locked host memory is needed for the overlap (pageable memory works
 * but copies synchronously).  beta == 0 never reads C.  Not for use inside
 * CUDA-graph capture.  Returns a sgemm_b200_status; after an error some
 * blocks of C may be updated. */
int sgemm_b200_host(int path, int m, int n, int k,
                    const float* alpha,
                    const float* A, int lda,
                    const float* B, int ldb,
                    const float* beta,
                    float* C, int ldc,
                    sgemm_b200_stream_t stream);

/* Block plan sgemm_b200_host uses for this problem when it does not take the
 * k-outer plan (sgemm_b200_host_plan_kouter; host-only): writes the
 * rows per band to *rows and the widths of up to max_chunks column chunks to
 * chunk_cols, and returns the number of chunks (m rows and one chunk of n
 * columns when it does not split), or a negated sgemm_b200_status. */
int sgemm_b200_host_plan(int path, int m, int n, int k, int reads_c, int* rows,
                         int* chunk_cols, int max_chunks);

/* Whether sgemm_b200_host takes its k-outer plan for this problem (host-only;
 * plain path, large problems, when the plan's timing model puts it at least
 * 3% ahead of the block plan above).  That plan streams A and B in k slices,
 * running a whole-C GEMM per slice as soon as it lands with the FP32 sums
 * carried between launches in device memory, then finishes the last k
 * columns row band by row band with alpha/beta applied, each band returning
 * while the next computes; slices start on whole 32-deep k blocks, so C has
 * the same bits.  Writes k values of the sliced phase to *k_outer (0: the
 * block plan runs), its slice count to *slices and the band height to *rows;
 * returns a sgemm_b200_status.  sgemm_b200_host_planned always runs the block
 * plan it is given.  No reference counterpart. */
int sgemm_b200_host_plan_kouter(int path, int m, int n, int k, int reads_c, int* k_outer,
                                int* slices, int* rows);

/* sgemm_b200_host with the caller's block plan instead of the built-in one:
 * bands of `rows` rows (the last takes the rest; at most 16 bands) times
 * `nchunks` (1..4) column chunks of the widths in chunk_cols, which must sum
 * to n.  Same result, bit for bit, for every valid plan; an invalid plan
 * returns SGEMM_B200_ERR_INVALID_ARG before any work. */
int sgemm_b200_host_planned(int path, int m, int n, int k,
                            const float* alpha,
                            const float* A, int lda,
                            const float* B, int ldb,
                            const float* beta,
                            float* C, int ldc,
                            int rows, const int* chunk_cols, int nchunks,
                            sgemm_b200_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Grouped persistent GEMM (no reference counterpart)                        */
/* ------------------------------------------------------------------------ */

typedef struct {
    int m, n, k;
    int lda, ldb, ldc;
    float alpha, beta;
    const float* A;
    const float* B;
    float* C;
} sgemm_b200_problem;

/* Opaque plan: problem table on the device, tile schedule, split-K choice per
 * problem, and (after the first launch) a captured CUDA graph. */
typedef struct sgemm_b200_grouped_plan sgemm_b200_grouped_plan;

/* Build a plan for `count` problems (host array, copied).  tuning_json may be
 * NULL (built-in choices) or a path written by sgemm_b200_autotune_grouped. */
int sgemm_b200_grouped_plan_create(sgemm_b200_grouped_plan** plan,
                                   const sgemm_b200_problem* problems, int count,
                                   const char* tuning_json);
/* One persistent launch over every problem of the plan on `stream`.
 * use_graph != 0 replays a CUDA graph captured on the first call.  A plan
 * holds its own work-ticket counters, so launches of one plan must not
 * overlap on the GPU: order them on one stream (distinct plans may run
 * concurrently). */
int sgemm_b200_grouped_plan_launch(sgemm_b200_grouped_plan* plan,
                                   sgemm_b200_stream_t stream, int use_graph);
/* Tiles and work items in the plan's schedule (for tests and reports). */
int sgemm_b200_grouped_plan_info(const sgemm_b200_grouped_plan* plan,
                                 int* tiles, int* work_items, int* grid_ctas);
void sgemm_b200_grouped_plan_destroy(sgemm_b200_grouped_plan* plan);

/* One-shot convenience: plan, launch once, synchronise, destroy. */
int sgemm_b200_grouped(const sgemm_b200_problem* problems, int count,
                       sgemm_b200_stream_t stream);

/* The baseline the grouped launch replaces: one sgemm_b200 call per problem,
 * in order, on `stream`. */
int sgemm_b200_grouped_sequential(const sgemm_b200_problem* problems, int count,
                                  sgemm_b200_stream_t stream);

/* Host-only schedule summary (no device needed): the tiles, work items and
 * split-K workspace bytes a plan for these problems would use with the given
 * tuning table (NULL = built-in choices, or when the table does not match). */
int sgemm_b200_grouped_schedule(const sgemm_b200_problem* problems, int count,
                                const char* tuning_json, int* tiles, int* work_items,
                                size_t* workspace_bytes);

/* Grouped split-precision GEMM (no reference counterpart): every problem of
 * the table -- C := alpha*A*B + beta*C, each with sgemm_b200's argument
 * meaning -- through one grouped pre-pass launch that writes all problems'
 * BF16 (path BF16X6) or TF32 (path TF32X3) planes, and one launch of a
 * persistent tcgen05 kernel over the 128 x 256 tiles of all problems
 * (per-problem tensor maps, longest tiles first).  Each problem's result
 * equals sgemm_b200_split's on its own, bit for bit.  Workspace for the
 * planes and the launch tables come stream-ordered from the library's pool
 * and are released after the kernels.  Problems with k == 0 run on the plain
 * path (C := beta*C).  Stream-ordered; returns without synchronising. */
int sgemm_b200_grouped_split(int path, const sgemm_b200_problem* problems, int count,
                             sgemm_b200_stream_t stream);

/* The baseline that launch replaces: one sgemm_b200_split call per problem,
 * in order, on `stream`. */
int sgemm_b200_grouped_split_sequential(int path, const sgemm_b200_problem* problems, int count,
                                        sgemm_b200_stream_t stream);

/* Size bucket (0..8) the tuning table keys a problem by: 3 classes of M*N
 * (< 256^2, < 1024^2, larger) x 3 classes of K (< 512, < 2048, larger). */
int sgemm_b200_grouped_bucket(int m, int n, int k);

/* Time the candidate tile/stage/split-K choices per size bucket on the current
 * device with the given problems and write the winners to json_path. */
int sgemm_b200_autotune_grouped(const sgemm_b200_problem* problems, int count,
                                const char* json_path);

/* ------------------------------------------------------------------------ */
/* Utilities                                                                 */
/* ------------------------------------------------------------------------ */

/* Distributions of the seeded counter-based generator. */
typedef enum {
    SGEMM_B200_DIST_UNIFORM_PM1 = 0,  /* uniform[-1, 1) */
    SGEMM_B200_DIST_UNIFORM_01 = 1,   /* uniform[0, 1)  (the reference's init_random) */
    SGEMM_B200_DIST_SIGNED_POW2 = 2   /* random sign * 2^e * uniform[1,2), e in [-10, 10] */
} sgemm_b200_dist;

/* Fill rows x cols (row stride ld) of a device matrix with value
 * f(seed, tag, row*cols + col) of the chosen distribution.  The same values
 * come out of the host generator in the oracle, bit for bit. */
int sgemm_b200_fill_random(float* X, int rows, int cols, int ld,
                           uint64_t seed, uint32_t tag, int dist,
                           sgemm_b200_stream_t stream);

/* Bytes the library's own stream-ordered memory pool on the current device
 * holds for live allocations (*used_bytes) and keeps reserved from the driver
 * (*reserved_bytes).  The pool backs the scratch the library allocates itself:
 * split workspaces when the caller passes none, packed copies of unaligned
 * operands, and the host-operand path's staging.  Both are 0 before any call
 * on the device has created the pool; the query never creates it. */
int sgemm_b200_pool_usage(size_t* used_bytes, size_t* reserved_bytes);

/* Reads and clears the device-side status word that bounded waits set on
 * expiry (SGEMM_B200_OK or SGEMM_B200_ERR_TIMEOUT).  Synchronises the device. */
int sgemm_b200_device_status(void);

/* Self-test of the failure path above (no reference counterpart): launches
 * one thread that waits, bounded by limit_us microseconds (1..10^7), on an
 * mbarrier phase that nothing completes -- the situation of a TMA copy or MMA
 * group that never lands -- and records SGEMM_B200_ERR_TIMEOUT in the status
 * word the way the GEMM kernels do.  The kernel then returns normally; after
 * `stream` completes, sgemm_b200_device_status() reports the timeout and the
 * device remains usable.  Returns the launch status. */
int sgemm_b200_selftest_wait_timeout(int limit_us, sgemm_b200_stream_t stream);

/* Status of the most recent call on this thread (used by sgemm(), which
 * returns void like the reference). */
int sgemm_b200_last_status(void);
const char* sgemm_b200_status_string(int status);

/* Detail of the most recent failure on the calling thread: the failing CUDA
 * call's error name and message, or the rejected tensor-map parameters; "" if
 * nothing has failed yet.  Not cleared by successful calls. */
const char* sgemm_b200_last_error_detail(void);

/* Library version string. */
const char* sgemm_b200_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SGEMM_B200_H */
