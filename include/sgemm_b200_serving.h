/*
 * sgemm_b200_serving.h — continuous-batching GEMM server (no reference
 * counterpart: the reference has no serving code).
 *
 * A server owns one device memory pool of `hbm_budget_bytes`.  Each request
 * is a GEMM C := alpha*A*B + beta*C whose operands the server allocates from
 * the pool when the request is admitted and keeps resident on the device
 * until the caller releases the request.  Admission is by memory: a request
 * waits in the arrival queue until its A, B and C fit in the pool, and is
 * refused (SGEMM_B200_ERR_REJECTED) if they could never fit.
 *
 * Continuous batching: admitted requests are grouped into batches as soon as
 * one of `slots` CUDA streams is free; each batch runs as one launch of the
 * persistent grouped kernel (plain path) or as one split-precision GEMM per
 * request (BF16X6 / TF32X3 paths) on that slot's stream.  Requests that
 * arrive while other batches are on the GPU are admitted as memory frees and
 * join the next batch, so batches overlap on the device.  Every request's
 * result is independent of the batch it lands in: the grouped kernel runs
 * the plain path's exact arithmetic per problem, and the split paths compute
 * each request alone.
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

/* Block until every submitted request has completed or been refused. */
int sgemm_b200_server_drain(sgemm_b200_server* server);

/* Result of a completed request (keep_results != 0): latency and the device
 * pointer of its C (row stride n), valid until released. */
int sgemm_b200_server_result(sgemm_b200_server* server, int64_t request_id, double* latency_ms,
                             const float** C, int* ldc, int* batch_size);
/* Copy a completed request's C (m x n, row-major, packed) to host memory. */
int sgemm_b200_server_read_result(sgemm_b200_server* server, int64_t request_id, float* host_out);
int sgemm_b200_server_release(sgemm_b200_server* server, int64_t request_id);

int sgemm_b200_server_get_stats(sgemm_b200_server* server, sgemm_b200_server_stats* out);

/* Copy the trace of the statistics window (run_poisson starts a new window):
 * up to `max` records of completed requests in completion order; *count
 * receives the number written.  A window keeps at most 1,048,576 records;
 * later completions still count in the statistics but are not traced. */
int sgemm_b200_server_get_trace(sgemm_b200_server* server, sgemm_b200_server_trace_record* out,
                                int max, int* count);

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
