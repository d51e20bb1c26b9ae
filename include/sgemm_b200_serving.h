/*
 * sgemm_b200_serving.h — continuous-batching GEMM server (no reference
 * counterpart: the reference has no serving code).
 *
 * A server owns one device memory pool of `hbm_budget_bytes`.  Each request
 * is a GEMM C := alpha*A*B + beta*C.  Its operands come from one of three
 * places, chosen by the submit call:
 *   - sgemm_b200_server_submit_device: the caller's own device matrices,
 *     used in place (the result lands in the caller's C);
 *   - sgemm_b200_server_submit_host: the caller's host matrices, copied into
 *     the pool when the request is admitted and C copied back after its batch,
 *     both inside the request's latency;
 *   - sgemm_b200_server_submit: matrices the server generates in the pool from
 *     a seed (for load tests that need no caller data).
 * Pool memory -- operands held in the pool, and the split paths' workspace --
 * is allocated when the request is admitted and kept until the request
 * completes (or, with keep_results, until the caller releases it).  Admission
 * is by memory: a request waits in the arrival queue until its pool memory
 * fits, and is refused (SGEMM_B200_ERR_REJECTED) if it could never fit.
 *
 * Continuous batching: admitted requests are grouped into batches as soon as
 * one of `slots` CUDA streams is free; each batch runs on that slot's stream
 * as one launch of the persistent grouped FFMA kernel (plain path) or as one
 * grouped split pre-pass plus one launch of the persistent grouped tcgen05
 * kernel (BF16X6 / TF32X3 paths).  Requests that
 * arrive while other batches are on the GPU are admitted as memory frees and
 * join the next batch, so batches overlap on the device.  Every request's
 * result is independent of the batch it lands in: the grouped kernel runs
 * the plain path's exact arithmetic per problem, and the grouped split kernel
 * computes each tile exactly as the single split GEMM does.
 *
 * Latency of a request = completion minus submission, on the host's steady
 * clock.  Completion is when the server's completion thread, which polls an
 * event recorded after each batch's last kernel, sees the batch finished.
 */
#ifndef SGEMM_B200_SERVING_H
#define SGEMM_B200_SERVING_H

#include <stddef.h>
#include <stdint.h>

#include "sgemm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sgemm_b200_server sgemm_b200_server;

typedef struct {
    size_t hbm_budget_bytes;  /* device pool size */
    int slots;                /* batches that may be in flight at once (streams) */
    int max_batch;            /* most requests in one batch */
    int path;                 /* sgemm_b200_path */
    int keep_results;         /* 0: free a request's memory when it completes */
    /* fault injection for tests (0 = off) */
    int inject_alloc_failure_every;  /* every Nth admission fails as out-of-memory */
    int inject_batch_delay_ms;       /* host delay before each batch launch */
} sgemm_b200_server_config;

typedef struct {
    int64_t submitted, completed, rejected, failed;
    int64_t batches;
    int max_batches_in_flight;     /* most batches seen on the GPU at once */
    int max_batch_size;
    double p50_ms, p99_ms, mean_ms, max_ms;  /* latency of completed requests */
    double gflops;                 /* completed FLOPs / (last completion - first submit) */
    double wall_s;
    size_t peak_pool_bytes;
    int64_t peak_waiting;          /* largest arrival-queue length seen */
    /* latency split at the batch launch: queue = submission to the host-side
     * launch of the request's batch, service = that launch to completion */
    double queue_p50_ms, queue_p99_ms, service_p50_ms, service_p99_ms;
} sgemm_b200_server_stats;

/* One completed request.  Times are host steady-clock milliseconds from the
 * first submission of the statistics window. */
typedef struct {
    int64_t request_id;
    int m, n, k;
    int batch_size;
    int64_t batch;     /* batch number within the window, from 1 */
    double submit_ms;  /* sgemm_b200_server_submit */
    double admit_ms;   /* operands allocated from the pool, generation enqueued */
    double launch_ms;  /* the batch's launch began on the host */
    double done_ms;    /* the completion thread saw the batch finished */
    /* the batch's span on the device (CUDA events after its operands are
     * ready and after its last kernel), ms from an event recorded at the
     * window's first submission; -1 when unavailable */
    double device_start_ms, device_end_ms;
} sgemm_b200_server_trace_record;

int sgemm_b200_server_create(sgemm_b200_server** server, const sgemm_b200_server_config* cfg);
/* Stop the server: requests that have not reached the GPU are cancelled (they
 * count as failed), batches in flight complete, then every resource is
 * released.  Waits for the server's own streams only. */
void sgemm_b200_server_destroy(sgemm_b200_server* server);

/* Submit one request.  The operands are allocated from the pool at admission
 * and filled from the seeded generator (uniform[-1, 1): A tag 1, B tag 2, C
 * tag 3 of `seed`).  Returns at once with the request id. */
int sgemm_b200_server_submit(sgemm_b200_server* server, int m, int n, int k, float alpha,
                             float beta, uint64_t seed, int64_t* request_id);

/* Submit C := alpha*A*B + beta*C on the caller's DEVICE matrices (on the
 * server's device; row-major, row strides lda >= k, ldb >= n, ldc >= n, the
 * meaning of sgemm_b200's arguments).  The matrices must be complete on the
 * device when this is called (the server does not wait on the caller's
 * streams).  Ownership stays with the caller: A and B must stay valid and
 * unchanged, and C must be neither read nor written, until the request has
 * completed (sgemm_b200_server_wait or _drain); C is then the result.  The
 * pool holds only the split paths' workspace.  Returns at once. */
int sgemm_b200_server_submit_device(sgemm_b200_server* server, int m, int n, int k,
                                    float alpha, const float* A, int lda, const float* B,
                                    int ldb, float beta, float* C, int ldc,
                                    int64_t* request_id);

/* Submit C := alpha*A*B + beta*C on the caller's HOST matrices (row-major,
 * strides as above).  At admission the server allocates A, B and C in its
 * pool and copies A, B (and C when beta != 0) in on its ingest stream; after
 * the request's batch it copies C back into the caller's C.  The request
 * completes when that copy has landed, so its latency includes both copies.
 * The buffers must stay valid and unchanged (C untouched) until completion;
 * page-locked memory lets the copies run asynchronously (pageable memory
 * works, but each copy then blocks the server's worker thread while it runs).
 * Returns at once. */
int sgemm_b200_server_submit_host(sgemm_b200_server* server, int m, int n, int k, float alpha,
                                  const float* A, int lda, const float* B, int ldb, float beta,
                                  float* C, int ldc, int64_t* request_id);

/* Block until one request has completed, failed or been refused; returns
 * SGEMM_B200_OK, SGEMM_B200_ERR_CUDA or SGEMM_B200_ERR_REJECTED and, when
 * completed, its latency.  Must not race with sgemm_b200_server_release of the
 * same request. */
int sgemm_b200_server_wait(sgemm_b200_server* server, int64_t request_id, double* latency_ms);

/* Block until every submitted request has completed or been refused. */
int sgemm_b200_server_drain(sgemm_b200_server* server);

/* Result of a completed request: latency and the device pointer and row
 * stride of its C -- the caller's own C for device requests, else the pool's
 * copy (kept only with keep_results != 0, valid until released; NULL once
 * the pool memory has been freed). */
int sgemm_b200_server_result(sgemm_b200_server* server, int64_t request_id, double* latency_ms,
                             const float** C, int* ldc, int* batch_size);
/* Copy a completed request's C (m x n) to host memory as packed rows: from
 * the device C (device requests, or pool copies that are kept) or from the
 * caller's host C (host requests). */
int sgemm_b200_server_read_result(sgemm_b200_server* server, int64_t request_id, float* host_out);
int sgemm_b200_server_release(sgemm_b200_server* server, int64_t request_id);

int sgemm_b200_server_get_stats(sgemm_b200_server* server, sgemm_b200_server_stats* out);

/* Copy the trace of the statistics window (run_poisson starts a new window):
 * up to `max` records of completed requests in completion order; *count
 * receives the number written.  A window keeps at most 1,048,576 records;
 * later completions still count in the statistics but are not traced. */
int sgemm_b200_server_get_trace(sgemm_b200_server* server, sgemm_b200_server_trace_record* out,
                                int max, int* count);

/* Device time of one request of shape m x n x k served alone through this
 * server's own batch launch (the same kernels, on one of its slot streams,
 * operands generated in its pool): the median of `reps` launches, as the
 * device span the trace records for served batches.  The server must be idle
 * (nothing queued or running, else SGEMM_B200_ERR_INVALID_ARG), and the
 * request's pool memory must fit (else SGEMM_B200_ERR_NO_MEMORY).  Used as the
 * floor a served request's latency is compared with. */
int sgemm_b200_server_isolated_ms(sgemm_b200_server* server, int m, int n, int k, int reps,
                                  double* ms);

/* Open-loop load: `n_requests` requests with exponential inter-arrival times
 * of mean 1/rate_per_s; 60% tall-skinny (M uniform in [16, 256], N = K =
 * 4096), 40% square (M = N = K log-uniform in [512, 4096], multiples of 8).
 * Blocks until all complete; fills `out`. */
int sgemm_b200_server_run_poisson(sgemm_b200_server* server, double rate_per_s, int n_requests,
                                  uint64_t seed, sgemm_b200_server_stats* out);

/* Host-only pieces, exposed for tests without a GPU. */
/* Draw the request mix: writes n (m, n, k) triples and inter-arrival gaps. */
int sgemm_b200_serving_workload(int n_requests, double rate_per_s, uint64_t seed, int* mnk,
                                double* gaps_s);
/* Offset pool (first fit, coalescing, 256-byte aligned) used for the budget. */
typedef struct sgemm_b200_pool sgemm_b200_pool;
sgemm_b200_pool* sgemm_b200_pool_create(size_t capacity);
void sgemm_b200_pool_destroy(sgemm_b200_pool* pool);
/* Returns the offset, or -1 when the request does not fit now. */
int64_t sgemm_b200_pool_alloc(sgemm_b200_pool* pool, size_t bytes);
int sgemm_b200_pool_free(sgemm_b200_pool* pool, int64_t offset);
size_t sgemm_b200_pool_used(const sgemm_b200_pool* pool);
size_t sgemm_b200_pool_largest_free(const sgemm_b200_pool* pool);

#ifdef __cplusplus
}
#endif

#endif /* SGEMM_B200_SERVING_H */
