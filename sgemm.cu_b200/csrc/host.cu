// host.cu — GEMM on operands that live in host memory.
//
// The reference has no such entry point: its callers copy A, B and C to the
// device with cudaMemcpy, call sgemm(), and copy C back (test.cu:70-80,
// benchmark.cu:69-73), so the PCIe transfers and the kernel run one after the
// other.  Here the library stages the operands through HBM itself and overlaps
// the three phases.  C is cut into blocks: row bands (at most 16, multiples of
// 128 rows) times column chunks (1..4, of planned widths); the blocks go
// column chunk by column chunk:
//
//   copy stream (H2D):  B[:, chunk j], then per row band b: A[b, :] (first
//                       chunk only) and, when beta != 0, C[b, chunk j]
//   compute streams:    block (b, j) runs on one of four compute streams as soon
//                       as its operands have landed, so a block's kernel
//                       overlaps its neighbours' copies and wave tails
//   copy stream (D2H):  C[b, chunk j] back to the host once computed
//
// Column chunks let the first kernel start after part of B instead of all
// of it; the chunk widths come from a small timing model of this pipeline
// (PCIe bandwidth and per-path GEMM rate measured on a B200), evaluated for
// even and uneven splits per call.  Every block is the same GEMM on a sub-matrix, issued
// through sgemm_b200_gemm(); each C element keeps its k-ordered accumulation,
// so the result is bit-identical to copying the whole matrices and calling the
// device entry point once.
//
// Device memory: A, B and C at 16-byte-aligned pitches, from the library's
// stream-ordered pool.  Host buffers should be page-locked (cudaMallocHost /
// cudaHostRegister): pageable memory gives the same result, but the driver
// then stages copies synchronously and nothing overlaps.  Device pointers are
// accepted too (the copies use cudaMemcpyDefault).
#include <algorithm>
#include <mutex>

#include "common.h"
#include "plain.h"

namespace sgb {
namespace host {

constexpr int kComputeStreams = 4;
constexpr int kMaxBands = 16;
constexpr int kMaxChunks = 4;
constexpr int kMaxBlocks = kMaxBands * kMaxChunks;

struct Engine {
    bool ready = false;
    cudaStream_t h2d = nullptr, d2h = nullptr, comp[kComputeStreams] = {};
    cudaEvent_t start = nullptr;
    cudaEvent_t b_in[kMaxChunks] = {}, in[kMaxBlocks] = {}, done[kMaxBlocks] = {};
    cudaEvent_t tail[2 + kComputeStreams] = {};
    std::mutex mu;  // one call at a time enqueues on the engine's streams and events
};

static Engine* engine() {
    constexpr int kMaxDevices = 64;
    static Engine engines[kMaxDevices];
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    Engine& e = engines[dev];
    if (!e.ready) {
        const unsigned sf = cudaStreamNonBlocking;
        const unsigned ef = cudaEventDisableTiming;
        bool ok = cudaStreamCreateWithFlags(&e.h2d, sf) == cudaSuccess &&
                  cudaStreamCreateWithFlags(&e.d2h, sf) == cudaSuccess &&
                  cudaEventCreateWithFlags(&e.start, ef) == cudaSuccess;
        for (int i = 0; ok && i < kComputeStreams; ++i)
            ok = cudaStreamCreateWithFlags(&e.comp[i], sf) == cudaSuccess;
        for (int i = 0; ok && i < kMaxChunks; ++i)
            ok = cudaEventCreateWithFlags(&e.b_in[i], ef) == cudaSuccess;
        for (int i = 0; ok && i < kMaxBlocks; ++i)
            ok = cudaEventCreateWithFlags(&e.in[i], ef) == cudaSuccess &&
                 cudaEventCreateWithFlags(&e.done[i], ef) == cudaSuccess;
        for (int i = 0; ok && i < 2 + kComputeStreams; ++i)
            ok = cudaEventCreateWithFlags(&e.tail[i], ef) == cudaSuccess;
        if (!ok) return nullptr;  // partially created handles live until exit
        e.ready = true;
    }
    return &e;
}

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Smallest block worth a kernel of its own: one 128 x 64 CTA tile per SM.
// With four compute streams, four such blocks in flight cover every resident
// CTA slot, so the timing model's "GEMMs run at full rate" stays true.
constexpr double kMinBlockElems = 148.0 * 128 * 64;

// Rows per band for blocks `cols` wide: at most kMaxBands bands, blocks of at
// least kMinBlockElems, a multiple of 128 rows (the tallest CTA tile), and
// bands of even height.
static int band_rows(int m, int cols) {
    const int r_min = static_cast<int>((kMinBlockElems + cols - 1) / cols);
    int r = std::max((m + kMaxBands - 1) / kMaxBands, r_min);
    r = (r + 127) / 128 * 128;
    if (r >= m) return m;
    const int bands = (m + r - 1) / r;
    r = ((m + bands - 1) / bands + 127) / 128 * 128;
    return std::min(m, r);
}

// A plan: row bands of `rows` rows (the last takes the rest) times up to
// kMaxChunks column chunks of the given widths (multiples of 128 but the
// last), taken chunk by chunk.
struct Plan {
    int rows;
    int nchunks;
    int cols[kMaxChunks];
};

// Timing model of the pipeline: one H2D queue, one D2H queue, and the GEMMs
// as one server at the path's rate.  Constants measured on a B200 (pinned
// host memory; GEMM rates at 8192^3).
static double model_ms(int path, int m, int k, bool read_c, const Plan& p) {
    constexpr double kPcieBytesPerS = 51e9;
    const double flops_per_s = path == SGEMM_B200_PATH_BF16X6   ? 225e12
                               : path == SGEMM_B200_PATH_TF32X3 ? 210e12
                                                                : 59e12;
    double t_h = 0, t_c = 0, t_d = 0;
    for (int j = 0; j < p.nchunks; ++j) {
        const double nc = p.cols[j];
        t_h += 4.0 * k * nc / kPcieBytesPerS;
        for (int r0 = 0; r0 < m; r0 += p.rows) {
            const double nr = std::min(p.rows, m - r0);
            if (j == 0) t_h += 4.0 * nr * k / kPcieBytesPerS;
            if (read_c) t_h += 4.0 * nr * nc / kPcieBytesPerS;
            t_c = std::max(t_c, t_h) + 2.0 * nr * nc * k / flops_per_s;
            t_d = std::max(t_d, t_c) + 4.0 * nr * nc / kPcieBytesPerS;
        }
    }
    return t_d * 1e3;
}

// Candidates: one chunk; 2..4 even chunks; and two or three uneven chunks
// with widths in steps of ~n/16.  An uneven plan with a wide first chunk
// gives each A band that arrives with the first chunk more work, so the
// phase in which A streams in stays compute-bound; narrow later chunks then
// start early.  Every chunk is at least 512 columns, and the rows per band
// keep every block at least kMinBlockElems.
Plan make_plan(int path, int m, int n, int k, bool read_c) {
    const double bytes = 4.0 * (double(m) * k + double(k) * n + double(m) * n * (read_c ? 2 : 1));
    Plan best{m, 1, {n}};
    if (bytes < 16.0 * (1 << 20)) return best;  // small: one block
    best.rows = band_rows(m, n);
    double best_t = model_ms(path, m, k, read_c, best);
    auto consider = [&](std::initializer_list<int> widths) {
        Plan p{0, 0, {}};
        int narrowest = n, used = 0;
        for (int w : widths) {
            if (w < 512) return;
            p.cols[p.nchunks++] = w;
            used += w;
            narrowest = std::min(narrowest, w);
        }
        if (n - used < 512) return;
        p.cols[p.nchunks++] = n - used;
        narrowest = std::min(narrowest, n - used);
        p.rows = band_rows(m, narrowest);
        const double t = model_ms(path, m, k, read_c, p);
        if (t < best_t * 0.98) {  // fewer, larger blocks unless clearly faster
            best_t = t;
            best = p;
        }
    };
    for (int s = 2; s <= 4; ++s) {  // even chunks
        const int c = (n + s - 1) / s / 128 * 128;
        if (s == 2) consider({c});
        if (s == 3) consider({c, c});
        if (s == 4) consider({c, c, c});
    }
    const int g = std::max(128, (n / 16 + 127) / 128 * 128);
    for (int a = g; a < n; a += g) {  // uneven: first chunk a, then b, then the rest
        consider({a});
        for (int b2 = g; a + b2 < n; b2 += g) consider({a, b2});
    }
    return best;
}

// ------------------------------------------------------- k-outer plan --
//
// Plain path only.  Phase 1 streams A and B in k slices (A[:, slice] and
// B[slice, :]) and runs a whole-C GEMM per slice as soon as its slice has
// landed, carrying the unscaled FP32 sums between launches in an m x n device
// buffer; phase 2 runs the last k2 = k - k1 columns band by band with the
// alpha/beta epilogue, each band returning to the host while the next
// computes.  The first GEMM starts after one thin slice instead of after a
// whole band of A and chunk of B, and C's return overlaps phase 2.  Slices
// start on multiples of 128 (whole 32-deep k blocks), so every element runs
// the same k-ordered FMA chain as in one launch: the same bits.
constexpr int kMaxSlices = 16;

struct KPlan {
    int k1;                   // phase 1 covers k in [0, k1); 0: not used
    int nslices;              // phase-1 slices: [cut[s], cut[s + 1])
    int cut[kMaxSlices + 1];
    int rows;                 // phase-2 band height
};

static double kouter_model_ms(int m, int n, int k, bool read_c, const KPlan& p) {
    constexpr double kPcieBytesPerS = 51e9, kFlopsPerS = 59e12;
    double t_h = 0, t_c = 0, t_d = 0;
    for (int s = 0; s < p.nslices; ++s) {
        const double ks = p.cut[s + 1] - p.cut[s];
        t_h += 4.0 * (double(m) + n) * ks / kPcieBytesPerS;
        t_c = std::max(t_c, t_h) + 2.0 * double(m) * n * ks / kFlopsPerS;
    }
    const double k2 = k - p.k1;
    t_h += 4.0 * k2 * n / kPcieBytesPerS;
    for (int r0 = 0; r0 < m; r0 += p.rows) {
        const double nr = std::min(p.rows, m - r0);
        t_h += 4.0 * nr * k2 / kPcieBytesPerS + (read_c ? 4.0 * nr * n / kPcieBytesPerS : 0.0);
        t_c = std::max(t_c, t_h) + 2.0 * nr * n * k2 / kFlopsPerS;
        t_d = std::max(t_d, t_c) + 4.0 * nr * n / kPcieBytesPerS;
    }
    return t_d * 1e3;
}

// Candidates: a thin first slice (256 or 512 columns), then slices of about
// 1024, and a phase 2 of 512..3072 columns in bands of the 2-D plan's height
// or of 512..2048 rows.  Returns the plan with k1 == 0 when none applies.
static KPlan make_kplan(int m, int n, int k, bool read_c, double* t_best) {
    KPlan best{};
    *t_best = 1e300;
    if (k < 2048 || m < 1024 || n < 1024) return best;
    for (int k2t : {512, 768, 1024, 1536, 2048, 3072}) {
        const int k1 = (k - k2t) / 128 * 128;
        if (k1 < 1024) continue;
        for (int first : {256, 512}) {
            KPlan p{};
            p.k1 = k1;
            p.cut[0] = 0;
            p.cut[1] = first;
            p.nslices = 1;
            const int rest = k1 - first;
            int parts = std::min(kMaxSlices - 1, (rest + 1023) / 1024);
            const int w = (rest / parts + 127) / 128 * 128;
            for (int c = first; c < k1 && p.nslices < kMaxSlices;) {
                const int next = (p.nslices == kMaxSlices - 1) ? k1 : std::min(k1, c + w);
                p.cut[++p.nslices] = next;
                c = next;
            }
            if (p.cut[p.nslices] != k1) continue;
            for (int rows : {band_rows(m, n), 512, 1024, 2048}) {
                if (rows >= m || (m + rows - 1) / rows > kMaxBands) continue;
                p.rows = rows;
                const double t = kouter_model_ms(m, n, k, read_c, p);
                if (t < *t_best) {
                    *t_best = t;
                    best = p;
                }
            }
        }
    }
    return best;
}

// The k-outer plan replaces the 2-D plan when the model puts it at least 3%
// ahead (plain path only: its kernels carry accumulators between launches).
static bool choose_kplan(int path, int m, int n, int k, bool read_c, const Plan& plan,
                         KPlan* out) {
    if (path != SGEMM_B200_PATH_PLAIN) return false;
    double t = 0;
    const KPlan kp = make_kplan(m, n, k, read_c, &t);
    if (kp.k1 <= 0 || !(t < 0.97 * model_ms(path, m, k, read_c, plan))) return false;
    *out = kp;
    return true;
}

// A plan is usable when its chunks cover n, its bands number at most
// kMaxBands and its blocks at most kMaxBlocks (the engine's event arrays).
static bool plan_ok(const Plan& p, int m, int n) {
    if (p.rows < 1 || p.nchunks < 1 || p.nchunks > kMaxChunks) return false;
    if ((m + p.rows - 1) / p.rows > kMaxBands) return false;
    long long cols = 0;
    for (int j = 0; j < p.nchunks; ++j) {
        if (p.cols[j] < 1) return false;
        cols += p.cols[j];
    }
    return cols == n;
}

// Streams: the H2D stream brings phase 1's slices in order, then B's last k2
// rows, then per band A's last k2 columns and (beta != 0) C; phase 1 runs on
// compute stream 0; phase 2's bands run on the four compute streams once
// phase 1 and their operands are done; the D2H stream returns each band.
static int run_kouter(int m, int n, int k, const float* alpha, const float* A, int lda,
                      const float* B, int ldb, const float* beta, float* C, int ldc,
                      cudaStream_t stream, const KPlan& kp) {
    Engine* eng = engine();
    if (!eng) return SGEMM_B200_ERR_CUDA;
    cudaMemPool_t pool = library_pool();
    if (!pool) return SGEMM_B200_ERR_CUDA;
    const bool read_c = *beta != 0.0f;
    const int bands = (m + kp.rows - 1) / kp.rows;
    if (kp.nslices < 1 || kp.nslices > kMaxSlices || bands > kMaxBands ||
        kp.nslices + bands > kMaxBlocks)
        return SGEMM_B200_ERR_INVALID_ARG;
    const int lda_d = (k + 3) / 4 * 4, ldb_d = (n + 3) / 4 * 4, ldc_d = (n + 3) / 4 * 4;
    const size_t a_bytes = align_up(sizeof(float) * (size_t)m * lda_d, 256);
    const size_t b_bytes = align_up(sizeof(float) * (size_t)k * ldb_d, 256);
    const size_t c_bytes = align_up(sizeof(float) * (size_t)m * ldc_d, 256);

    std::lock_guard<std::mutex> lock(eng->mu);
    void* base = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&base, a_bytes + b_bytes + 2 * c_bytes, pool, stream);
    if (e != cudaSuccess) return cuda_status(e);
    char* p8 = static_cast<char*>(base);
    float* dA = reinterpret_cast<float*>(p8);
    float* dB = reinterpret_cast<float*>(p8 + a_bytes);
    float* dC = reinterpret_cast<float*>(p8 + a_bytes + b_bytes);
    float* dAcc = reinterpret_cast<float*>(p8 + a_bytes + b_bytes + c_bytes);

    int status = SGEMM_B200_OK;
    auto ok = [&](cudaError_t r) {
        if (r != cudaSuccess && status == SGEMM_B200_OK) status = cuda_status(r);
        return status == SGEMM_B200_OK;
    };
    auto gemm_ok = [&](int g) {
        if (g != SGEMM_B200_OK && status == SGEMM_B200_OK) status = g;
        return status == SGEMM_B200_OK;
    };
    const size_t f = sizeof(float);
    cudaStream_t all[2 + kComputeStreams];
    all[0] = eng->h2d;
    all[1] = eng->d2h;
    for (int i = 0; i < kComputeStreams; ++i) all[2 + i] = eng->comp[i];
    if (ok(cudaEventRecord(eng->start, stream)))
        for (cudaStream_t s : all) ok(cudaStreamWaitEvent(s, eng->start, 0));

    // phase 1: whole-C GEMMs over the k slices, sums carried in dAcc
    for (int s = 0; s < kp.nslices && status == SGEMM_B200_OK; ++s) {
        const int c0 = kp.cut[s], ks = kp.cut[s + 1] - kp.cut[s];
        if (!ok(cudaMemcpy2DAsync(dA + c0, f * lda_d, A + c0, f * lda, f * ks, m,
                                  cudaMemcpyDefault, eng->h2d)) ||
            !ok(cudaMemcpy2DAsync(dB + (size_t)c0 * ldb_d, f * ldb_d, B + (size_t)c0 * ldb,
                                  f * ldb, f * n, ks, cudaMemcpyDefault, eng->h2d)) ||
            !ok(cudaEventRecord(eng->in[s], eng->h2d)) ||
            !ok(cudaStreamWaitEvent(eng->comp[0], eng->in[s], 0)))
            break;
        if (!gemm_ok(plain_launch_acc(-1, m, n, ks, *alpha, dA + c0, lda_d,
                                      dB + (size_t)c0 * ldb_d, ldb_d, *beta, dC, ldc_d,
                                      s > 0 ? dAcc : nullptr, dAcc, ldc_d, eng->comp[0])))
            break;
    }
    ok(cudaEventRecord(eng->b_in[1], eng->comp[0]));  // phase 1 done
    // phase 2: the last k2 columns band by band, alpha/beta applied, C returned
    const int k1 = kp.k1, k2 = k - kp.k1;
    if (status == SGEMM_B200_OK &&
        ok(cudaMemcpy2DAsync(dB + (size_t)k1 * ldb_d, f * ldb_d, B + (size_t)k1 * ldb, f * ldb,
                             f * n, k2, cudaMemcpyDefault, eng->h2d)))
        ok(cudaEventRecord(eng->b_in[0], eng->h2d));
    for (int b = 0; b < bands && status == SGEMM_B200_OK; ++b) {
        const int r0 = b * kp.rows, nr = std::min(kp.rows, m - r0);
        const int ev = kp.nslices + b;
        cudaStream_t cs = eng->comp[b % kComputeStreams];
        if (!ok(cudaMemcpy2DAsync(dA + (size_t)r0 * lda_d + k1, f * lda_d,
                                  A + (size_t)r0 * lda + k1, f * lda, f * k2, nr,
                                  cudaMemcpyDefault, eng->h2d)))
            break;
        if (read_c && !ok(cudaMemcpy2DAsync(dC + (size_t)r0 * ldc_d, f * ldc_d,
                                            C + (size_t)r0 * ldc, f * ldc, f * n, nr,
                                            cudaMemcpyDefault, eng->h2d)))
            break;
        if (!ok(cudaEventRecord(eng->in[ev], eng->h2d)) ||
            !ok(cudaStreamWaitEvent(cs, eng->b_in[1], 0)) ||
            !ok(cudaStreamWaitEvent(cs, eng->b_in[0], 0)) ||
            !ok(cudaStreamWaitEvent(cs, eng->in[ev], 0)))
            break;
        if (!gemm_ok(plain_launch_acc(-1, nr, n, k2, *alpha, dA + (size_t)r0 * lda_d + k1, lda_d,
                                      dB + (size_t)k1 * ldb_d, ldb_d, *beta,
                                      dC + (size_t)r0 * ldc_d, ldc_d, dAcc + (size_t)r0 * ldc_d,
                                      nullptr, ldc_d, cs)))
            break;
        if (!ok(cudaEventRecord(eng->done[b], cs)) ||
            !ok(cudaStreamWaitEvent(eng->d2h, eng->done[b], 0)))
            break;
        ok(cudaMemcpy2DAsync(C + (size_t)r0 * ldc, f * ldc, dC + (size_t)r0 * ldc_d, f * ldc_d,
                             f * n, nr, cudaMemcpyDefault, eng->d2h));
    }
    for (int i = 0; i < 2 + kComputeStreams; ++i) {
        if (cudaEventRecord(eng->tail[i], all[i]) == cudaSuccess)
            cudaStreamWaitEvent(stream, eng->tail[i], 0);
    }
    cudaFreeAsync(base, stream);
    return status;
}

static int run(int path, int m, int n, int k, const float* alpha, const float* A, int lda,
               const float* B, int ldb, const float* beta, float* C, int ldc,
               cudaStream_t stream, const Plan* forced) {
    Engine* eng = engine();
    if (!eng) return SGEMM_B200_ERR_CUDA;
    cudaMemPool_t pool = library_pool();
    if (!pool) return SGEMM_B200_ERR_CUDA;

    const bool read_c = *beta != 0.0f;  // beta == 0: C is written, never read
    const Plan plan = forced ? *forced : make_plan(path, m, n, k, read_c);
    KPlan kp{};
    if (!forced && choose_kplan(path, m, n, k, read_c, plan, &kp))
        return run_kouter(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream, kp);
    const int bands = (m + plan.rows - 1) / plan.rows;
    // Device pitches: rows start on 16 bytes, so the TMA kernels take every block.
    const int lda_d = (k + 3) / 4 * 4, ldb_d = (n + 3) / 4 * 4, ldc_d = (n + 3) / 4 * 4;
    const size_t a_bytes = align_up(sizeof(float) * (size_t)m * lda_d, 256);
    const size_t b_bytes = align_up(sizeof(float) * (size_t)k * ldb_d, 256);
    const size_t c_bytes = align_up(sizeof(float) * (size_t)m * ldc_d, 256);

    std::lock_guard<std::mutex> lock(eng->mu);
    void* base = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&base, a_bytes + b_bytes + c_bytes, pool, stream);
    if (e != cudaSuccess) return cuda_status(e);
    float* dA = static_cast<float*>(base);
    float* dB = reinterpret_cast<float*>(static_cast<char*>(base) + a_bytes);
    float* dC = reinterpret_cast<float*>(static_cast<char*>(base) + a_bytes + b_bytes);

    int status = SGEMM_B200_OK;
    auto ok = [&](cudaError_t r) {
        if (r != cudaSuccess && status == SGEMM_B200_OK) status = cuda_status(r);
        return status == SGEMM_B200_OK;
    };
    const size_t f = sizeof(float);
    cudaStream_t all[2 + kComputeStreams];
    all[0] = eng->h2d;
    all[1] = eng->d2h;
    for (int i = 0; i < kComputeStreams; ++i) all[2 + i] = eng->comp[i];
    // Everything below starts after the caller's prior work and the allocation.
    if (ok(cudaEventRecord(eng->start, stream)))
        for (cudaStream_t s : all) ok(cudaStreamWaitEvent(s, eng->start, 0));

    int blk = 0;
    for (int j = 0, c0 = 0; j < plan.nchunks && status == SGEMM_B200_OK; c0 += plan.cols[j++]) {
        const int nc = plan.cols[j];
        if (k > 0 && ok(cudaMemcpy2DAsync(dB + c0, f * ldb_d, B + c0, f * ldb, f * nc, k,
                                          cudaMemcpyDefault, eng->h2d)))
            ok(cudaEventRecord(eng->b_in[j], eng->h2d));
        for (int b = 0; b < bands && status == SGEMM_B200_OK; ++b, ++blk) {
            const int r0 = b * plan.rows, nr = std::min(plan.rows, m - r0);
            cudaStream_t cs = eng->comp[blk % kComputeStreams];
            // H2D: this block's operands (A's band only with the first chunk).
            if (j == 0 && k > 0 &&
                !ok(cudaMemcpy2DAsync(dA + (size_t)r0 * lda_d, f * lda_d, A + (size_t)r0 * lda,
                                      f * lda, f * k, nr, cudaMemcpyDefault, eng->h2d)))
                break;
            if (read_c &&
                !ok(cudaMemcpy2DAsync(dC + (size_t)r0 * ldc_d + c0, f * ldc_d,
                                      C + (size_t)r0 * ldc + c0, f * ldc, f * nc, nr,
                                      cudaMemcpyDefault, eng->h2d)))
                break;
            if (!ok(cudaEventRecord(eng->in[blk], eng->h2d))) break;
            // Compute.
            if (k > 0 && !ok(cudaStreamWaitEvent(cs, eng->b_in[j], 0))) break;
            if (!ok(cudaStreamWaitEvent(cs, eng->in[blk], 0))) break;
            const int g = sgemm_b200_gemm(path, nr, nc, k, alpha, dA + (size_t)r0 * lda_d, lda_d,
                                          dB + c0, ldb_d, beta, dC + (size_t)r0 * ldc_d + c0,
                                          ldc_d, reinterpret_cast<sgemm_b200_stream_t>(cs));
            if (g != SGEMM_B200_OK) {
                status = g;
                break;
            }
            if (!ok(cudaEventRecord(eng->done[blk], cs))) break;
            // D2H.
            if (ok(cudaStreamWaitEvent(eng->d2h, eng->done[blk], 0)))
                ok(cudaMemcpy2DAsync(C + (size_t)r0 * ldc + c0, f * ldc,
                                     dC + (size_t)r0 * ldc_d + c0, f * ldc_d, f * nc, nr,
                                     cudaMemcpyDefault, eng->d2h));
        }
    }
    // Join: the caller's stream waits for whatever was enqueued on the
    // engine's streams (also after an error), then releases the staging memory.
    for (int i = 0; i < 2 + kComputeStreams; ++i) {
        if (cudaEventRecord(eng->tail[i], all[i]) == cudaSuccess)
            cudaStreamWaitEvent(stream, eng->tail[i], 0);
    }
    cudaFreeAsync(base, stream);
    return status;
}

}  // namespace host
}  // namespace sgb

extern "C" int sgemm_b200_host(int path, int m, int n, int k, const float* alpha, const float* A,
                               int lda, const float* B, int ldb, const float* beta, float* C,
                               int ldc, sgemm_b200_stream_t stream) {
    int s = sgb::check_gemm_args(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    if (s == SGEMM_B200_OK && path != SGEMM_B200_PATH_PLAIN && path != SGEMM_B200_PATH_BF16X6 &&
        path != SGEMM_B200_PATH_TF32X3)
        s = SGEMM_B200_ERR_INVALID_ARG;
    if (s == SGEMM_B200_OK && m > 0 && n > 0) {
        if (!sgb::device_is_sm100())
            s = SGEMM_B200_ERR_UNSUPPORTED;
        else
            s = sgb::host::run(path, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                               sgb::as_stream(stream), nullptr);
    }
    sgb::set_last_status(s);
    return s;
}

extern "C" int sgemm_b200_host_planned(int path, int m, int n, int k, const float* alpha,
                                       const float* A, int lda, const float* B, int ldb,
                                       const float* beta, float* C, int ldc, int rows,
                                       const int* chunk_cols, int nchunks,
                                       sgemm_b200_stream_t stream) {
    int s = sgb::check_gemm_args(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    if (s == SGEMM_B200_OK && path != SGEMM_B200_PATH_PLAIN && path != SGEMM_B200_PATH_BF16X6 &&
        path != SGEMM_B200_PATH_TF32X3)
        s = SGEMM_B200_ERR_INVALID_ARG;
    sgb::host::Plan p{rows, nchunks, {}};
    if (s == SGEMM_B200_OK && m > 0 && n > 0) {
        if (!chunk_cols || nchunks < 1 || nchunks > sgb::host::kMaxChunks) {
            s = SGEMM_B200_ERR_INVALID_ARG;
        } else {
            for (int j = 0; j < nchunks; ++j) p.cols[j] = chunk_cols[j];
            if (!sgb::host::plan_ok(p, m, n)) s = SGEMM_B200_ERR_INVALID_ARG;
        }
    }
    if (s == SGEMM_B200_OK && m > 0 && n > 0) {
        if (!sgb::device_is_sm100())
            s = SGEMM_B200_ERR_UNSUPPORTED;
        else
            s = sgb::host::run(path, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                               sgb::as_stream(stream), &p);
    }
    sgb::set_last_status(s);
    return s;
}

extern "C" int sgemm_b200_host_plan_kouter(int path, int m, int n, int k, int reads_c,
                                           int* k_outer, int* slices, int* rows) {
    if (m <= 0 || n <= 0 || k < 0 || !k_outer || !slices || !rows)
        return SGEMM_B200_ERR_INVALID_ARG;
    const sgb::host::Plan p = sgb::host::make_plan(path, m, n, k, reads_c != 0);
    sgb::host::KPlan kp{};
    if (sgb::host::choose_kplan(path, m, n, k, reads_c != 0, p, &kp)) {
        *k_outer = kp.k1;
        *slices = kp.nslices;
        *rows = kp.rows;
    } else {
        *k_outer = 0;
        *slices = 0;
        *rows = 0;
    }
    return SGEMM_B200_OK;
}

extern "C" int sgemm_b200_host_plan(int path, int m, int n, int k, int reads_c, int* rows,
                                    int* chunk_cols, int max_chunks) {
    if (m <= 0 || n <= 0 || k < 0 || !rows || !chunk_cols || max_chunks < 1)
        return -SGEMM_B200_ERR_INVALID_ARG;
    const sgb::host::Plan p = sgb::host::make_plan(path, m, n, k, reads_c != 0);
    *rows = p.rows;
    for (int j = 0; j < p.nchunks && j < max_chunks; ++j) chunk_cols[j] = p.cols[j];
    return p.nchunks;
}
