// serving.cu — continuous-batching GEMM server (no reference counterpart; the
// reference has no serving code).  See include/sgemm_b200_serving.h for the
// contract.
//
// Threads and streams:
//  - the caller's thread submits requests (or run_poisson submits them on an
//    open-loop schedule);
//  - one worker thread admits requests in arrival order while their operands
//    fit in the pool (generating them on an ingest stream), forms a batch
//    whenever one of `slots` streams is free, and launches it: one persistent
//    grouped FFMA kernel (plain path) or one grouped split pre-pass and one
//    persistent grouped tcgen05 kernel (split paths), followed by an event on
//    the slot's stream;
//  - one completion thread polls the events of the batches in flight
//    (cudaEventQuery, about every 20 us, asleep while nothing is in flight),
//    stamps the completion time of a finished batch's requests and hands the
//    slot back.  Polling rather than a host callback (cudaLaunchHostFunc):
//    on B200 the driver's callback thread was measured to start callbacks
//    ~40 ms after their batch had finished on the device, once or twice per
//    few thousand batches, which set the p99 of whole runs.
// Requests that arrive while batches run are admitted as memory frees and
// join the next batch; with two or more slots, batches overlap on the GPU.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/sgemm_b200_serving.h"
#include "common.h"
#include "grouped.h"
#include "rng.h"
#include "split.h"

// ------------------------------------------------------------------- pool --

// First-fit offset allocator with coalescing over [0, capacity); 256-byte
// granularity.  Pure host bookkeeping: the server maps offsets onto one
// device allocation.
struct sgemm_b200_pool {
    size_t capacity = 0;
    size_t used = 0;
    std::map<size_t, size_t> free_;  // offset -> size
    std::map<size_t, size_t> live_;  // offset -> size
};

namespace sgb {
namespace serving {

constexpr size_t kAlign = 256;
constexpr size_t kMaxTrace = size_t(1) << 20;  // trace records kept per window

static size_t round_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

static int64_t pool_alloc(sgemm_b200_pool* p, size_t bytes) {
    const size_t need = round_up(std::max<size_t>(bytes, 1));
    for (auto it = p->free_.begin(); it != p->free_.end(); ++it) {
        if (it->second < need) continue;
        const size_t off = it->first, size = it->second;
        p->free_.erase(it);
        if (size > need) p->free_[off + need] = size - need;
        p->live_[off] = need;
        p->used += need;
        return (int64_t)off;
    }
    return -1;
}

static int pool_free(sgemm_b200_pool* p, int64_t offset) {
    auto it = p->live_.find((size_t)offset);
    if (it == p->live_.end()) return SGEMM_B200_ERR_INVALID_ARG;
    size_t off = it->first, size = it->second;
    p->live_.erase(it);
    p->used -= size;
    auto next = p->free_.lower_bound(off);
    if (next != p->free_.end() && off + size == next->first) {
        size += next->second;
        next = p->free_.erase(next);
    }
    if (next != p->free_.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == off) {
            prev->second += size;
            return SGEMM_B200_OK;
        }
    }
    p->free_[off] = size;
    return SGEMM_B200_OK;
}

// ---------------------------------------------------------------- workload --

// Uniform double in [0, 1) from the counter-based generator.
static double unit(uint64_t key, uint64_t i) {
    return (double)(rng_mix(key + i) >> 11) * (1.0 / 9007199254740992.0);
}

static void workload(int n, double rate, uint64_t seed, int* mnk, double* gaps) {
    const uint64_t key = rng_key(seed, 0x5e4u);
    for (int i = 0; i < n; ++i) {
        const double u0 = unit(key, 4ull * i), u1 = unit(key, 4ull * i + 1);
        const double u2 = unit(key, 4ull * i + 2), u3 = unit(key, 4ull * i + 3);
        if (u0 < 0.6) {  // tall-skinny: M uniform in [16, 256], N = K = 4096
            mnk[3 * i] = 16 + (int)std::floor(u1 * 241.0);
            mnk[3 * i + 1] = 4096;
            mnk[3 * i + 2] = 4096;
        } else {  // square: log-uniform in [512, 4096], multiple of 8
            const double s = std::exp(std::log(512.0) + u1 * (std::log(4096.0) - std::log(512.0)));
            const int v = std::max(512, std::min(4096, (int)std::lround(s / 8.0) * 8));
            mnk[3 * i] = mnk[3 * i + 1] = mnk[3 * i + 2] = v;
        }
        (void)u2;
        gaps[i] = rate > 0 ? -std::log(1.0 - u3) / rate : 0.0;  // exponential inter-arrival
    }
}

// ------------------------------------------------------------------ server --

using Clock = std::chrono::steady_clock;

static double secs(Clock::time_point t) {
    return std::chrono::duration<double>(t.time_since_epoch()).count();
}

enum ReqState { kWaiting, kAdmitted, kRunning, kDone, kRejected, kFailed };

// Where a request's operands come from:
//  kGenerated  the server generates them in its pool (seeded, uniform[-1, 1))
//  kDevice     the caller's device matrices, used in place (C written in place)
//  kHost       the caller's host matrices: copied into the pool at admission,
//              C copied back after the batch (both inside the request's latency)
enum ReqKind { kGenerated = 0, kDevice = 1, kHost = 2 };

struct Request {
    int64_t id = 0;
    int kind = kGenerated;
    int m = 0, n = 0, k = 0;
    int lda = 0, ldb = 0, ldc = 0;  // of A, B, C as the kernels read them
    float alpha = 1, beta = 0;
    uint64_t seed = 0;
    size_t bytes = 0, ws_bytes = 0;
    int64_t off = -1;
    float *A = nullptr, *B = nullptr, *C = nullptr;  // device operands the batch uses
    const float* hA = nullptr;                       // kHost: the caller's buffers
    const float* hB = nullptr;
    float* hC = nullptr;
    int h_lda = 0, h_ldb = 0, h_ldc = 0;
    void* ws = nullptr;
    double t_submit = 0, t_admit = 0, t_launch = 0, t_done = 0;
    int state = kWaiting;
    int batch_size = 0;
    int64_t batch = 0;
    bool auto_release = false;
    cudaEvent_t ready = nullptr;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_end = nullptr;  // device span of the current batch
    bool error = false;  // the batch's end event reported an error
    bool busy = false;
    std::vector<Request*> batch;
    grouped::Arena arena;      // plain path: grouped FFMA launches
    split::Arena split_arena;  // split paths: grouped tcgen05 launches
};

struct Server;

struct Server {
    sgemm_b200_server_config cfg;
    uint8_t* d_pool = nullptr;
    sgemm_b200_pool pool;
    cudaStream_t ingest = nullptr;
    cudaEvent_t epoch = nullptr;  // recorded on `ingest` at the window's first submission
    bool epoch_set = false;
    std::vector<Slot> slots;
    std::vector<int> polling;  // slots whose batch is on the GPU, oldest first
    int device = 0;

    std::mutex mu;
    std::condition_variable cv, cv_drain, cv_poll;
    std::deque<Request*> arrivals;
    std::deque<Request*> ready;
    std::deque<int> finished_slots;
    std::unordered_map<int64_t, Request*> all;
    std::thread worker, completer;
    bool stop = false;
    int64_t next_id = 1;
    int64_t outstanding = 0;  // submitted and not yet done / rejected / failed
    int64_t admissions = 0;

    // stats
    std::vector<double> latencies_ms, queue_ms, service_ms;
    std::vector<sgemm_b200_server_trace_record> trace;
    double flops_done = 0, t_first_submit = -1, t_last_done = 0;
    int64_t submitted = 0, completed = 0, rejected = 0, failed = 0, batches = 0;
    int in_flight = 0, max_in_flight = 0, max_batch_seen = 0;
    size_t peak_pool = 0;
    int64_t peak_waiting = 0;
};

// Completion thread: polls the end events of the batches in flight.
static void completer_loop(Server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lock(s->mu);
    while (true) {
        if (s->polling.empty()) {
            if (s->stop && s->outstanding == 0) break;
            s->cv_poll.wait_for(lock, std::chrono::milliseconds(50));
            continue;
        }
        const std::vector<int> slots = s->polling;
        lock.unlock();
        std::vector<int> done;
        std::vector<bool> ok;
        for (int si : slots) {
            const cudaError_t q = cudaEventQuery(s->slots[si].ev_end);
            if (q == cudaErrorNotReady) continue;
            done.push_back(si);
            ok.push_back(q == cudaSuccess);
        }
        const double t = secs(Clock::now());
        lock.lock();
        for (size_t i = 0; i < done.size(); ++i) {
            const int si = done[i];
            s->slots[si].error = !ok[i];
            for (Request* r : s->slots[si].batch) r->t_done = t;
            s->polling.erase(std::find(s->polling.begin(), s->polling.end(), si));
            s->finished_slots.push_back(si);
        }
        if (!done.empty()) {
            s->cv.notify_all();
            continue;
        }
        lock.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(20));
        lock.lock();
    }
}

// Pool bytes of one request: its operands (unless they are the caller's
// device matrices) and the split workspace.
static size_t request_bytes(int path, int kind, int m, int n, int k, size_t* ws) {
    const size_t a = round_up((size_t)m * k * 4), b = round_up((size_t)k * n * 4),
                 c = round_up((size_t)m * n * 4);
    *ws = path == SGEMM_B200_PATH_PLAIN ? 0
                                        : round_up(sgemm_b200_split_workspace_size(path, m, n, k));
    return (kind == kDevice ? 0 : a + b + c) + *ws;
}

// Called with the lock held.
static void finish_slot(Server* s, int si) {
    Slot& sl = s->slots[si];
    // the batch's device span on the device clock, from the window's epoch
    float g0 = -1.f, g1 = -1.f;
    if (s->epoch_set && (cudaEventElapsedTime(&g0, s->epoch, sl.ev_start) != cudaSuccess ||
                         cudaEventElapsedTime(&g1, s->epoch, sl.ev_end) != cudaSuccess)) {
        g0 = g1 = -1.f;
        cudaGetLastError();  // a failed query must not surface at this thread's next launch
    }
    for (Request* r : sl.batch) {
        if (r->ready) {
            cudaEventDestroy(r->ready);
            r->ready = nullptr;
        }
        if (sl.error) {  // the device reported an error for the batch
            r->state = kFailed;
            ++s->failed;
            --s->outstanding;
            if (r->auto_release) {
                pool_free(&s->pool, r->off);
                r->off = -1;
            }
            continue;
        }
        r->state = kDone;
        s->latencies_ms.push_back((r->t_done - r->t_submit) * 1e3);
        s->queue_ms.push_back((r->t_launch - r->t_submit) * 1e3);
        s->service_ms.push_back((r->t_done - r->t_launch) * 1e3);
        if (s->trace.size() < kMaxTrace) {
            const double t0 = s->t_first_submit;
            s->trace.push_back(sgemm_b200_server_trace_record{
                r->id, r->m, r->n, r->k, r->batch_size, r->batch, (r->t_submit - t0) * 1e3,
                (r->t_admit - t0) * 1e3, (r->t_launch - t0) * 1e3, (r->t_done - t0) * 1e3,
                (double)g0, (double)g1});
        }
        s->flops_done += 2.0 * r->m * (double)r->n * r->k;
        s->t_last_done = std::max(s->t_last_done, r->t_done);
        ++s->completed;
        --s->outstanding;
        if (r->auto_release) {
            pool_free(&s->pool, r->off);
            r->off = -1;
        }
    }
    sl.batch.clear();
    sl.busy = false;
    sl.error = false;
    --s->in_flight;
    s->cv_drain.notify_all();  // sgemm_b200_server_wait waits for single requests
}

// Admit arrivals in order while they fit (called with the lock held).
static void admit(Server* s) {
    while (!s->arrivals.empty()) {
        Request* r = s->arrivals.front();
        int64_t off = -1;
        const bool injected = s->cfg.inject_alloc_failure_every > 0 &&
                              (s->admissions + 1) % s->cfg.inject_alloc_failure_every == 0;
        if (!injected) off = pool_alloc(&s->pool, r->bytes);
        if (injected) {
            // An allocation failure the pool could not recover from: refuse.
            ++s->admissions;
            s->arrivals.pop_front();
            r->state = kFailed;
            ++s->failed;
            --s->outstanding;
            continue;
        }
        if (off < 0) break;  // wait for memory to free (keeps arrival order)
        ++s->admissions;
        s->arrivals.pop_front();
        r->off = off;
        uint8_t* base = s->d_pool + off;
        const size_t a = round_up((size_t)r->m * r->k * 4), b = round_up((size_t)r->k * r->n * 4),
                     c = round_up((size_t)r->m * r->n * 4);
        s->peak_pool = std::max(s->peak_pool, s->pool.used);
        if (r->kind == kDevice) {
            // The caller's matrices, complete on the device before submission:
            // nothing to wait for (ready stays null).
            r->ws = r->ws_bytes ? base : nullptr;
        } else {
            r->A = reinterpret_cast<float*>(base);
            r->B = reinterpret_cast<float*>(base + a);
            r->C = reinterpret_cast<float*>(base + a + b);
            r->ws = r->ws_bytes ? base + a + b + c : nullptr;
            if (r->kind == kGenerated) {
                // Operands arrive: generated on the device, resident from here on.
                sgemm_b200_fill_random(r->A, r->m, r->k, r->k, r->seed, 1,
                                       SGEMM_B200_DIST_UNIFORM_PM1, s->ingest);
                sgemm_b200_fill_random(r->B, r->k, r->n, r->n, r->seed, 2,
                                       SGEMM_B200_DIST_UNIFORM_PM1, s->ingest);
                sgemm_b200_fill_random(r->C, r->m, r->n, r->n, r->seed, 3,
                                       SGEMM_B200_DIST_UNIFORM_PM1, s->ingest);
            } else {
                // The caller's host matrices cross into the pool (C only if read).
                cudaMemcpy2DAsync(r->A, (size_t)r->k * 4, r->hA, (size_t)r->h_lda * 4,
                                  (size_t)r->k * 4, r->m, cudaMemcpyHostToDevice, s->ingest);
                cudaMemcpy2DAsync(r->B, (size_t)r->n * 4, r->hB, (size_t)r->h_ldb * 4,
                                  (size_t)r->n * 4, r->k, cudaMemcpyHostToDevice, s->ingest);
                if (r->beta != 0.0f)
                    cudaMemcpy2DAsync(r->C, (size_t)r->n * 4, r->hC, (size_t)r->h_ldc * 4,
                                      (size_t)r->n * 4, r->m, cudaMemcpyHostToDevice, s->ingest);
            }
            cudaEventCreateWithFlags(&r->ready, cudaEventDisableTiming);
            cudaEventRecord(r->ready, s->ingest);
        }
        r->t_admit = secs(Clock::now());
        r->state = kAdmitted;
        s->ready.push_back(r);
    }
}

// Shutdown: requests that have not reached the GPU fail instead of waiting,
// so that destroy ends once the batches in flight complete (called with the
// lock held).  Admitted requests' operand fills may still be running on the
// ingest stream; destroy synchronises it before freeing the pool.
static void cancel_pending(Server* s) {
    auto cancel = [&](Request* r) {
        if (r->ready) {
            cudaEventDestroy(r->ready);
            r->ready = nullptr;
        }
        if (r->off >= 0 && r->auto_release) {
            pool_free(&s->pool, r->off);
            r->off = -1;
        }
        r->state = kFailed;
        ++s->failed;
        --s->outstanding;
    };
    for (Request* r : s->arrivals) cancel(r);
    for (Request* r : s->ready) cancel(r);
    s->arrivals.clear();
    s->ready.clear();
}

static int launch_batch(Server* s, int si) {
    Slot& sl = s->slots[si];
    if (s->cfg.inject_batch_delay_ms > 0)
        std::this_thread::sleep_for(std::chrono::milliseconds(s->cfg.inject_batch_delay_ms));
    for (Request* r : sl.batch)
        if (r->ready) cudaStreamWaitEvent(sl.stream, r->ready, 0);
    int st = cuda_status(cudaEventRecord(sl.ev_start, sl.stream));
    if (st == SGEMM_B200_OK && s->cfg.path == SGEMM_B200_PATH_PLAIN) {
        std::vector<sgemm_b200_problem> probs(sl.batch.size());
        for (size_t i = 0; i < sl.batch.size(); ++i) {
            const Request* r = sl.batch[i];
            probs[i] = sgemm_b200_problem{r->m,     r->n,    r->k, r->lda, r->ldb, r->ldc,
                                          r->alpha, r->beta, r->A, r->B,   r->C};
        }
        st = grouped::arena_launch(&sl.arena, probs.data(), (int)probs.size(), sl.stream);
    } else if (st == SGEMM_B200_OK) {
        // one grouped pre-pass and one persistent tcgen05 launch for the batch
        std::vector<sgemm_b200_problem> probs(sl.batch.size());
        std::vector<void*> ws(sl.batch.size());
        for (size_t i = 0; i < sl.batch.size(); ++i) {
            const Request* r = sl.batch[i];
            probs[i] = sgemm_b200_problem{r->m,     r->n,    r->k, r->lda, r->ldb, r->ldc,
                                          r->alpha, r->beta, r->A, r->B,   r->C};
            ws[i] = r->ws;
        }
        st = split::grouped_launch(&sl.split_arena, s->cfg.path, probs.data(), ws.data(),
                                   (int)probs.size(), sl.stream);
    }
    // Results the caller wants in host memory go back before the batch counts
    // as complete.
    for (Request* r : sl.batch) {
        if (st != SGEMM_B200_OK) break;
        if (r->kind == kHost)
            st = cuda_status(cudaMemcpy2DAsync(r->hC, (size_t)r->h_ldc * 4, r->C, (size_t)r->ldc * 4,
                                               (size_t)r->n * 4, r->m, cudaMemcpyDeviceToHost,
                                               sl.stream));
    }
    if (st == SGEMM_B200_OK) st = cuda_status(cudaEventRecord(sl.ev_end, sl.stream));
    return st;
}

static void worker_loop(Server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lock(s->mu);
    while (true) {
        while (!s->finished_slots.empty()) {
            const int si = s->finished_slots.front();
            s->finished_slots.pop_front();
            finish_slot(s, si);
        }
        if (s->stop) cancel_pending(s);
        admit(s);
        s->peak_waiting = std::max<int64_t>(s->peak_waiting, (int64_t)s->arrivals.size());
        int free_slot = -1;
        for (size_t i = 0; i < s->slots.size(); ++i)
            if (!s->slots[i].busy) {
                free_slot = (int)i;
                break;
            }
        // With a batch already on the GPU, a new batch takes only requests whose
        // operands are in place: one whose generation is still running would
        // hold the slot, and the GPU, behind it.  Generation runs in admission
        // order on one stream, so those requests are a prefix of the queue.
        // With the GPU idle, a batch takes what is queued and its launch waits
        // on the device.
        bool wait_for_operands = false;
        if (free_slot >= 0 && !s->ready.empty()) {
            Slot& sl = s->slots[free_slot];
            const bool gpu_idle = s->in_flight == 0;
            while (!s->ready.empty() && (int)sl.batch.size() < s->cfg.max_batch) {
                Request* r = s->ready.front();
                if (!gpu_idle && r->ready && cudaEventQuery(r->ready) == cudaErrorNotReady) break;
                s->ready.pop_front();
                r->state = kRunning;
                sl.batch.push_back(r);
            }
            wait_for_operands = sl.batch.empty();
        }
        if (free_slot >= 0 && !s->slots[free_slot].batch.empty()) {
            Slot& sl = s->slots[free_slot];
            sl.busy = true;
            ++s->in_flight;
            ++s->batches;
            const double t_launch = secs(Clock::now());
            for (Request* r : sl.batch) {
                r->batch_size = (int)sl.batch.size();
                r->batch = s->batches;
                r->t_launch = t_launch;
            }
            s->max_in_flight = std::max(s->max_in_flight, s->in_flight);
            s->max_batch_seen = std::max(s->max_batch_seen, (int)sl.batch.size());
            lock.unlock();
            const int st = launch_batch(s, free_slot);
            // A launch that failed part-way may have left work on the slot's
            // stream that still reads or writes the batch's memory: let it
            // finish before that memory can go to another request.
            if (st != SGEMM_B200_OK) cudaStreamSynchronize(sl.stream);
            lock.lock();
            if (st != SGEMM_B200_OK) {
                // Fail the batch's requests.
                for (Request* r : sl.batch) {
                    r->state = kFailed;
                    ++s->failed;
                    --s->outstanding;
                    if (r->ready) {
                        cudaEventDestroy(r->ready);
                        r->ready = nullptr;
                    }
                    if (r->auto_release) {
                        pool_free(&s->pool, r->off);
                        r->off = -1;
                    }
                }
                sl.batch.clear();
                sl.busy = false;
                --s->in_flight;
            } else {
                s->polling.push_back(free_slot);
                s->cv_poll.notify_one();
            }
            continue;
        }
        s->cv_drain.notify_all();  // drain and per-request waiters re-check
        if (s->stop && s->outstanding == 0) break;
        if (wait_for_operands)
            s->cv.wait_for(lock, std::chrono::microseconds(20));
        else
            s->cv.wait_for(lock, std::chrono::milliseconds(2));
    }
}

}  // namespace serving
}  // namespace sgb

struct sgemm_b200_server {
    sgb::serving::Server s;
};

using sgb::serving::Request;
using sgb::serving::Server;

extern "C" sgemm_b200_pool* sgemm_b200_pool_create(size_t capacity) {
    auto* p = new sgemm_b200_pool();
    p->capacity = capacity / sgb::serving::kAlign * sgb::serving::kAlign;
    if (p->capacity) p->free_[0] = p->capacity;
    return p;
}
extern "C" void sgemm_b200_pool_destroy(sgemm_b200_pool* p) { delete p; }
extern "C" int64_t sgemm_b200_pool_alloc(sgemm_b200_pool* p, size_t bytes) {
    return p ? sgb::serving::pool_alloc(p, bytes) : -1;
}
extern "C" int sgemm_b200_pool_free(sgemm_b200_pool* p, int64_t off) {
    return p ? sgb::serving::pool_free(p, off) : SGEMM_B200_ERR_INVALID_ARG;
}
extern "C" size_t sgemm_b200_pool_used(const sgemm_b200_pool* p) { return p ? p->used : 0; }
extern "C" size_t sgemm_b200_pool_largest_free(const sgemm_b200_pool* p) {
    size_t best = 0;
    if (p)
        for (const auto& kv : p->free_) best = std::max(best, kv.second);
    return best;
}

extern "C" int sgemm_b200_serving_workload(int n_requests, double rate, uint64_t seed, int* mnk,
                                           double* gaps) {
    if (n_requests < 0 || !mnk || !gaps || rate < 0) return SGEMM_B200_ERR_INVALID_ARG;
    sgb::serving::workload(n_requests, rate, seed, mnk, gaps);
    return SGEMM_B200_OK;
}

extern "C" int sgemm_b200_server_create(sgemm_b200_server** out,
                                        const sgemm_b200_server_config* cfg) {
    if (!out || !cfg || cfg->slots < 1 || cfg->max_batch < 1 || cfg->hbm_budget_bytes == 0 ||
        cfg->path < 0 || cfg->path > 2)
        return SGEMM_B200_ERR_INVALID_ARG;
    if (!sgb::device_is_sm100()) return SGEMM_B200_ERR_UNSUPPORTED;
    auto* srv = new sgemm_b200_server();
    Server* s = &srv->s;
    s->cfg = *cfg;
    cudaGetDevice(&s->device);
    s->pool.capacity = cfg->hbm_budget_bytes / sgb::serving::kAlign * sgb::serving::kAlign;
    s->pool.free_[0] = s->pool.capacity;
    cudaError_t e = cudaMalloc(&s->d_pool, s->pool.capacity);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->ingest, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&s->epoch);
    s->slots.resize(cfg->slots);
    for (int i = 0; i < cfg->slots && e == cudaSuccess; ++i) {
        e = cudaStreamCreateWithFlags(&s->slots[i].stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreate(&s->slots[i].ev_start);
        if (e == cudaSuccess) e = cudaEventCreate(&s->slots[i].ev_end);
    }
    if (e != cudaSuccess) {
        for (auto& sl : s->slots) {
            if (sl.stream) cudaStreamDestroy(sl.stream);
            if (sl.ev_start) cudaEventDestroy(sl.ev_start);
            if (sl.ev_end) cudaEventDestroy(sl.ev_end);
        }
        if (s->epoch) cudaEventDestroy(s->epoch);
        if (s->ingest) cudaStreamDestroy(s->ingest);
        cudaFree(s->d_pool);
        delete srv;
        return sgb::cuda_status(e);
    }
    s->worker = std::thread(sgb::serving::worker_loop, s);
    s->completer = std::thread(sgb::serving::completer_loop, s);
    *out = srv;
    return SGEMM_B200_OK;
}

namespace sgb {
namespace serving {

// Queue a filled-in request (shape, kind, operands); assigns its id.
static int submit(Server* s, Request* r, int64_t* id) {
    r->bytes = request_bytes(s->cfg.path, r->kind, r->m, r->n, r->k, &r->ws_bytes);
    r->t_submit = secs(Clock::now());
    std::lock_guard<std::mutex> lock(s->mu);
    r->auto_release = s->cfg.keep_results == 0;
    r->id = s->next_id++;
    s->all[r->id] = r;
    if (id) *id = r->id;
    ++s->submitted;
    if (s->t_first_submit < 0) {
        s->t_first_submit = r->t_submit;
        s->epoch_set = cudaEventRecord(s->epoch, s->ingest) == cudaSuccess;
    }
    if (r->bytes > s->pool.capacity) {  // could never fit: refuse now
        r->state = kRejected;
        ++s->rejected;
        return SGEMM_B200_ERR_REJECTED;
    }
    ++s->outstanding;
    s->arrivals.push_back(r);
    s->cv.notify_all();
    return SGEMM_B200_OK;
}

}  // namespace serving
}  // namespace sgb

extern "C" int sgemm_b200_server_submit(sgemm_b200_server* srv, int m, int n, int k, float alpha,
                                        float beta, uint64_t seed, int64_t* id) {
    if (!srv || m <= 0 || n <= 0 || k <= 0) return SGEMM_B200_ERR_INVALID_ARG;
    auto* r = new Request();
    r->kind = sgb::serving::kGenerated;
    r->m = m;
    r->n = n;
    r->k = k;
    r->lda = k;
    r->ldb = n;
    r->ldc = n;
    r->alpha = alpha;
    r->beta = beta;
    r->seed = seed;
    return sgb::serving::submit(&srv->s, r, id);
}

extern "C" int sgemm_b200_server_submit_device(sgemm_b200_server* srv, int m, int n, int k,
                                               float alpha, const float* A, int lda,
                                               const float* B, int ldb, float beta, float* C,
                                               int ldc, int64_t* id) {
    if (!srv || m <= 0 || n <= 0 || k <= 0 || !A || !B || !C || lda < k || ldb < n || ldc < n)
        return SGEMM_B200_ERR_INVALID_ARG;
    auto* r = new Request();
    r->kind = sgb::serving::kDevice;
    r->m = m;
    r->n = n;
    r->k = k;
    r->lda = lda;
    r->ldb = ldb;
    r->ldc = ldc;
    r->alpha = alpha;
    r->beta = beta;
    r->A = const_cast<float*>(A);
    r->B = const_cast<float*>(B);
    r->C = C;
    return sgb::serving::submit(&srv->s, r, id);
}

extern "C" int sgemm_b200_server_submit_host(sgemm_b200_server* srv, int m, int n, int k,
                                             float alpha, const float* A, int lda, const float* B,
                                             int ldb, float beta, float* C, int ldc,
                                             int64_t* id) {
    if (!srv || m <= 0 || n <= 0 || k <= 0 || !A || !B || !C || lda < k || ldb < n || ldc < n)
        return SGEMM_B200_ERR_INVALID_ARG;
    auto* r = new Request();
    r->kind = sgb::serving::kHost;
    r->m = m;
    r->n = n;
    r->k = k;
    r->lda = k;  // packed in the pool
    r->ldb = n;
    r->ldc = n;
    r->alpha = alpha;
    r->beta = beta;
    r->hA = A;
    r->hB = B;
    r->hC = C;
    r->h_lda = lda;
    r->h_ldb = ldb;
    r->h_ldc = ldc;
    return sgb::serving::submit(&srv->s, r, id);
}

extern "C" int sgemm_b200_server_wait(sgemm_b200_server* srv, int64_t id, double* latency_ms) {
    if (!srv) return SGEMM_B200_ERR_INVALID_ARG;
    Server* s = &srv->s;
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return SGEMM_B200_ERR_INVALID_ARG;
    Request* r = it->second;
    s->cv.notify_all();
    s->cv_drain.wait(lock, [&] {
        return r->state == sgb::serving::kDone || r->state == sgb::serving::kFailed ||
               r->state == sgb::serving::kRejected;
    });
    if (latency_ms) *latency_ms = (r->t_done - r->t_submit) * 1e3;
    return r->state == sgb::serving::kDone       ? SGEMM_B200_OK
           : r->state == sgb::serving::kRejected ? SGEMM_B200_ERR_REJECTED
                                                 : SGEMM_B200_ERR_CUDA;
}

extern "C" int sgemm_b200_server_drain(sgemm_b200_server* srv) {
    if (!srv) return SGEMM_B200_ERR_INVALID_ARG;
    Server* s = &srv->s;
    std::unique_lock<std::mutex> lock(s->mu);
    s->cv.notify_all();
    s->cv_drain.wait(lock, [&] { return s->outstanding == 0; });
    return s->failed ? SGEMM_B200_ERR_CUDA : SGEMM_B200_OK;
}

extern "C" int sgemm_b200_server_result(sgemm_b200_server* srv, int64_t id, double* latency_ms,
                                        const float** C, int* ldc, int* batch_size) {
    if (!srv) return SGEMM_B200_ERR_INVALID_ARG;
    Server* s = &srv->s;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return SGEMM_B200_ERR_INVALID_ARG;
    Request* r = it->second;
    if (r->state == sgb::serving::kRejected) return SGEMM_B200_ERR_REJECTED;
    if (r->state != sgb::serving::kDone) return SGEMM_B200_ERR_CUDA;
    if (latency_ms) *latency_ms = (r->t_done - r->t_submit) * 1e3;
    // the caller's own C (device requests), else the pool's copy while it is kept
    const bool device_c = r->kind == sgb::serving::kDevice || r->off >= 0;
    if (C) *C = device_c ? r->C : nullptr;
    if (ldc) *ldc = r->ldc;
    if (batch_size) *batch_size = r->batch_size;
    return SGEMM_B200_OK;
}

extern "C" int sgemm_b200_server_read_result(sgemm_b200_server* srv, int64_t id, float* host_out) {
    if (!srv || !host_out) return SGEMM_B200_ERR_INVALID_ARG;
    Server* s = &srv->s;
    const float* C = nullptr;
    const float* hC = nullptr;
    int m = 0, n = 0, ldc = 0;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        auto it = s->all.find(id);
        if (it == s->all.end()) return SGEMM_B200_ERR_INVALID_ARG;
        Request* r = it->second;
        if (r->state != sgb::serving::kDone) return SGEMM_B200_ERR_INVALID_ARG;
        m = r->m;
        n = r->n;
        if (r->kind == sgb::serving::kHost) {
            hC = r->hC;  // the result is already in the caller's host C
            ldc = r->h_ldc;
        } else {
            if (r->kind == sgb::serving::kGenerated && r->off < 0)
                return SGEMM_B200_ERR_INVALID_ARG;  // released with its pool memory
            C = r->C;
            ldc = r->ldc;
        }
    }
    if (hC) {
        for (int i = 0; i < m; ++i)
            std::memcpy(host_out + (size_t)i * n, hC + (size_t)i * ldc, sizeof(float) * n);
        return SGEMM_B200_OK;
    }
    return sgb::cuda_status(cudaMemcpy2D(host_out, sizeof(float) * n, C, sizeof(float) * ldc,
                                         sizeof(float) * n, m, cudaMemcpyDeviceToHost));
}

extern "C" int sgemm_b200_server_release(sgemm_b200_server* srv, int64_t id) {
    if (!srv) return SGEMM_B200_ERR_INVALID_ARG;
    Server* s = &srv->s;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return SGEMM_B200_ERR_INVALID_ARG;
    Request* r = it->second;
    if (r->state != sgb::serving::kDone && r->state != sgb::serving::kRejected &&
        r->state != sgb::serving::kFailed)
        return SGEMM_B200_ERR_INVALID_ARG;  // still queued or on the GPU
    if (r->off >= 0) sgb::serving::pool_free(&s->pool, r->off);
    delete r;
    s->all.erase(it);
    s->cv.notify_all();
    return SGEMM_B200_OK;
}

extern "C" int sgemm_b200_server_isolated_ms(sgemm_b200_server* srv, int m, int n, int k,
                                             int reps, double* ms) {
    if (!srv || !ms || m <= 0 || n <= 0 || k <= 0 || reps < 1) return SGEMM_B200_ERR_INVALID_ARG;
    Server* s = &srv->s;
    Request r;
    r.kind = sgb::serving::kGenerated;
    r.m = m;
    r.n = n;
    r.k = k;
    r.lda = k;
    r.ldb = n;
    r.ldc = n;
    r.alpha = 1.0f;
    r.beta = 0.0f;
    r.bytes = sgb::serving::request_bytes(s->cfg.path, r.kind, m, n, k, &r.ws_bytes);
    int si = -1;
    {
        // Take a free slot while nothing is queued or running, so the
        // measurement has the GPU to itself and the worker leaves the slot alone.
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->outstanding != 0 || s->in_flight != 0) return SGEMM_B200_ERR_INVALID_ARG;
        for (size_t i = 0; i < s->slots.size(); ++i)
            if (!s->slots[i].busy) {
                si = (int)i;
                break;
            }
        if (si < 0) return SGEMM_B200_ERR_INVALID_ARG;
        r.off = sgb::serving::pool_alloc(&s->pool, r.bytes);
        if (r.off < 0) return SGEMM_B200_ERR_NO_MEMORY;
        s->slots[si].busy = true;
    }
    sgb::serving::Slot& sl = s->slots[si];
    uint8_t* base = s->d_pool + r.off;
    const size_t a = sgb::serving::round_up((size_t)m * k * 4),
                 b = sgb::serving::round_up((size_t)k * n * 4),
                 c = sgb::serving::round_up((size_t)m * n * 4);
    r.A = reinterpret_cast<float*>(base);
    r.B = reinterpret_cast<float*>(base + a);
    r.C = reinterpret_cast<float*>(base + a + b);
    r.ws = r.ws_bytes ? base + a + b + c : nullptr;
    int st = sgemm_b200_fill_random(r.A, m, k, k, 1, 1, SGEMM_B200_DIST_UNIFORM_PM1, sl.stream);
    if (st == SGEMM_B200_OK)
        st = sgemm_b200_fill_random(r.B, k, n, n, 1, 2, SGEMM_B200_DIST_UNIFORM_PM1, sl.stream);
    std::vector<float> t;
    sl.batch.assign(1, &r);
    // one untimed launch, then `reps` timed ones: the batch's device span, as
    // the trace records it for served batches
    for (int i = 0; i <= reps && st == SGEMM_B200_OK; ++i) {
        st = sgb::serving::launch_batch(s, si);
        if (st == SGEMM_B200_OK) st = sgb::cuda_status(cudaEventSynchronize(sl.ev_end));
        float x = 0;
        if (st == SGEMM_B200_OK && i > 0)
            st = sgb::cuda_status(cudaEventElapsedTime(&x, sl.ev_start, sl.ev_end));
        if (i > 0) t.push_back(x);
    }
    if (st != SGEMM_B200_OK) cudaStreamSynchronize(sl.stream);
    {
        std::lock_guard<std::mutex> lock(s->mu);
        sl.batch.clear();
        sl.busy = false;
        sgb::serving::pool_free(&s->pool, r.off);
        s->cv.notify_all();
    }
    if (st != SGEMM_B200_OK) return st;
    std::sort(t.begin(), t.end());
    *ms = t[t.size() / 2];
    return SGEMM_B200_OK;
}

extern "C" int sgemm_b200_server_get_stats(sgemm_b200_server* srv, sgemm_b200_server_stats* out) {
    if (!srv || !out) return SGEMM_B200_ERR_INVALID_ARG;
    Server* s = &srv->s;
    std::lock_guard<std::mutex> lock(s->mu);
    sgemm_b200_server_stats st{};
    st.submitted = s->submitted;
    st.completed = s->completed;
    st.rejected = s->rejected;
    st.failed = s->failed;
    st.batches = s->batches;
    st.max_batches_in_flight = s->max_in_flight;
    st.max_batch_size = s->max_batch_seen;
    // nearest-rank percentile of a sorted sample
    auto pct = [](const std::vector<double>& v, double q) {
        const size_t i = std::min(v.size() - 1, (size_t)std::ceil(q * v.size()) - 1);
        return v[i];
    };
    std::vector<double> l = s->latencies_ms, qu = s->queue_ms, sv = s->service_ms;
    std::sort(l.begin(), l.end());
    std::sort(qu.begin(), qu.end());
    std::sort(sv.begin(), sv.end());
    if (!l.empty()) {
        st.p50_ms = pct(l, 0.50);
        st.p99_ms = pct(l, 0.99);
        double sum = 0;
        for (double v : l) sum += v;
        st.mean_ms = sum / l.size();
        st.max_ms = l.back();
        st.queue_p50_ms = pct(qu, 0.50);
        st.queue_p99_ms = pct(qu, 0.99);
        st.service_p50_ms = pct(sv, 0.50);
        st.service_p99_ms = pct(sv, 0.99);
    }
    st.wall_s = s->t_first_submit >= 0 ? s->t_last_done - s->t_first_submit : 0;
    st.gflops = st.wall_s > 0 ? s->flops_done / st.wall_s * 1e-9 : 0;
    st.peak_pool_bytes = s->peak_pool;
    st.peak_waiting = s->peak_waiting;
    *out = st;
    return SGEMM_B200_OK;
}

extern "C" int sgemm_b200_server_get_trace(sgemm_b200_server* srv,
                                           sgemm_b200_server_trace_record* out, int max,
                                           int* count) {
    if (!srv || !count || max < 0 || (max > 0 && !out)) return SGEMM_B200_ERR_INVALID_ARG;
    Server* s = &srv->s;
    std::lock_guard<std::mutex> lock(s->mu);
    const int n = (int)std::min<size_t>(s->trace.size(), (size_t)max);
    std::copy(s->trace.begin(), s->trace.begin() + n, out);
    *count = n;
    return SGEMM_B200_OK;
}

extern "C" int sgemm_b200_server_run_poisson(sgemm_b200_server* srv, double rate, int n,
                                             uint64_t seed, sgemm_b200_server_stats* out) {
    if (!srv || n < 0 || rate <= 0) return SGEMM_B200_ERR_INVALID_ARG;
    Server* s = &srv->s;
    std::vector<int> mnk(3 * (size_t)n);
    std::vector<double> gaps(n);
    sgb::serving::workload(n, rate, seed, mnk.data(), gaps.data());
    {
        // this run's statistics start fresh
        std::lock_guard<std::mutex> lock(s->mu);
        s->latencies_ms.clear();
        s->queue_ms.clear();
        s->service_ms.clear();
        s->trace.clear();
        s->flops_done = 0;
        s->t_first_submit = -1;
        s->epoch_set = false;
        s->t_last_done = 0;
        s->submitted = s->completed = s->rejected = s->failed = s->batches = 0;
        s->max_in_flight = s->max_batch_seen = 0;
        s->peak_waiting = 0;
    }
    int keep;
    {
        // an open-loop run releases results as they complete
        std::lock_guard<std::mutex> lock(s->mu);
        keep = s->cfg.keep_results;
        s->cfg.keep_results = 0;
    }
    auto t = sgb::serving::Clock::now();
    std::vector<int64_t> ids;
    for (int i = 0; i < n; ++i) {
        t += std::chrono::duration_cast<sgb::serving::Clock::duration>(
            std::chrono::duration<double>(gaps[i]));
        std::this_thread::sleep_until(t);
        int64_t id = 0;
        sgemm_b200_server_submit(srv, mnk[3 * i], mnk[3 * i + 1], mnk[3 * i + 2], 1.0f, 0.0f,
                                 seed * 1000003ull + i, &id);
        ids.push_back(id);
    }
    const int d = sgemm_b200_server_drain(srv);
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->cfg.keep_results = keep;
    }
    for (int64_t id : ids) sgemm_b200_server_release(srv, id);
    if (out) sgemm_b200_server_get_stats(srv, out);
    return d;
}

extern "C" void sgemm_b200_server_destroy(sgemm_b200_server* srv) {
    if (!srv) return;
    Server* s = &srv->s;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    s->cv_poll.notify_all();
    if (s->worker.joinable()) s->worker.join();
    if (s->completer.joinable()) s->completer.join();
    // The server's own streams only; other work on the device is not waited for.
    if (s->ingest) cudaStreamSynchronize(s->ingest);
    for (auto& sl : s->slots)
        if (sl.stream) cudaStreamSynchronize(sl.stream);
    for (auto& sl : s->slots) {
        sgb::grouped::arena_release(&sl.arena);
        sgb::split::arena_release(&sl.split_arena);
        if (sl.stream) cudaStreamDestroy(sl.stream);
        if (sl.ev_start) cudaEventDestroy(sl.ev_start);
        if (sl.ev_end) cudaEventDestroy(sl.ev_end);
    }
    if (s->epoch) cudaEventDestroy(s->epoch);
    if (s->ingest) cudaStreamDestroy(s->ingest);
    for (auto& kv : s->all) {
        if (kv.second->ready) cudaEventDestroy(kv.second->ready);
        delete kv.second;
    }
    cudaFree(s->d_pool);
    delete srv;
}
