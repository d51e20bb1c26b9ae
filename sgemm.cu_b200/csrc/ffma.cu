// ffma.cu — plain-path kernel configurations, dispatch and the C ABI entry
// points that replace the reference's sgemm() (src/sgemm.cuh:19-48).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "common.h"
#include "ffma_kernel.cuh"
#include "plain.h"

namespace sgb {
namespace ffma {

// Compiled configurations (the public config id is the position in kConfigs).
//   tile      warps  thread tile  stages  loader   resident CTAs/SM
using C0 = Cfg<128, 256, 4, 2, 16, 4, kLoaderTma, 1>;        // 8 warps, 192 KB smem, 1/SM
using C1 = Cfg<128, 128, 4, 2, 8, 3, kLoaderTma, 2>;         // 8 warps,  96 KB, 2/SM
using C2 = Cfg<128, 128, 4, 1, 16, 3, kLoaderTma, 2>;        // 4 warps,  96 KB, 2/SM
using C3 = Cfg<64, 128, 2, 2, 8, 4, kLoaderTma, 2>;          // 4 warps,  96 KB, 2/SM
using C4 = Cfg<64, 64, 2, 1, 8, 4, kLoaderTma, 3>;           // 2 warps,  64 KB, 3/SM
using C5 = Cfg<64, 128, 2, 2, 8, 3, kLoaderTma, 3>;          // 4 warps,  72 KB, 3/SM
using C6 = Cfg<128, 64, 4, 1, 8, 3, kLoaderTma, 3>;          // 4 warps,  72 KB, 3/SM
// Small tiles with 8 x 4 threads, for problems that leave most SMs idle with
// the tiles above (shared memory limits them to 3 and 4 CTAs/SM).
using S0 = Cfg<64, 64, 2, 2, 4, 4, kLoaderTma, 4>;         // 4 warps,  64 KB
using S1 = Cfg<32, 64, 1, 2, 4, 4, kLoaderTma, 6>;         // 2 warps,  48 KB
using C8 = Cfg<128, 256, 4, 2, 16, 4, kLoaderAsync4, 1>;
using C9 = Cfg<128, 128, 4, 2, 8, 3, kLoaderAsync4, 2>;
using C11 = Cfg<64, 128, 2, 2, 8, 4, kLoaderAsync4, 2>;
using C12 = Cfg<64, 64, 2, 1, 8, 4, kLoaderAsync4, 3>;
using C14 = Cfg<128, 64, 4, 1, 8, 3, kLoaderAsync4, 3>;
// The 128 x 64 tile with twice the warps (8 x 4 threads): for problems that
// are a single partial wave, where each busy SM holds one tile and four warps
// cannot hide the shared-memory and barrier latency.
using W0 = Cfg<128, 64, 4, 2, 4, 3, kLoaderTma, 3>;        // 8 warps,  72 KB
using W1 = Cfg<128, 64, 4, 2, 4, 4, kLoaderTma, 2>;        // 8 warps,  96 KB
// The best large tile with a producer warp (per-stage empty mbarriers, no CTA
// barrier in the main loop).
using P0 = Cfg<128, 64, 4, 1, 8, 3, kLoaderTma, 3, 8, 1>;  // 4+1 warps, 72 KB
using P1 = Cfg<128, 64, 4, 1, 8, 4, kLoaderTma, 2, 8, 1>;  // 4+1 warps, 96 KB
// A 28 x 256 tile of four warps side by side, 7 x 8 outputs per thread, with a
// producer warp: a 1024 x 1024 output is 37 x 4 = 148 tiles, one per SM, each
// thread doing 56 FMAs per k step where the 128 x 64 tile (128 tiles, 20 SMs
// idle) does 64.  With 4 stages one CTA fits an SM; with 3, two do (2048^3:
// 592 tiles, two full waves of eight compute warps per SM).
using T0 = Cfg<28, 256, 1, 4, 8, 4, kLoaderTma, 1, 8, 1, 7>;  // 4+1 warps, 145 KB, 1/SM
using T3 = Cfg<28, 256, 1, 4, 8, 3, kLoaderTma, 2, 8, 1, 7>;  // 4+1 warps, 109 KB, 2/SM

struct ConfigDesc {
    const char* name;
    int bm, bn, threads, smem, loader;
    float efficiency;  // relative per-SM throughput when the grid fills the GPU
    // relative throughput used instead when the whole problem is one partial
    // wave with a single CTA on the busiest SM (a lone CTA per SM); 0: the
    // configuration's full-wave efficiency
    float lone;
    void (*kernel)(const CUtensorMap, const CUtensorMap, const Params);
};

template <class C>
constexpr ConfigDesc describe(const char* name, float eff, float lone = 0.0f) {
    return ConfigDesc{name, C::BM, C::BN, C::THREADS, C::SMEM_BYTES, C::LOADER, eff, lone,
                      &ffma_gemm_kernel<C>};
}

// Efficiencies: relative per-SM throughput of a full wave, normalised to the
// best configuration of the same loader (TMA: tma_128x64_w4_t8x8_s3;
// cp.async: cpa_128x256_w8_t8x16_s4).  The large tiles were measured at
// 8192^3 / 16384^3 (the 8 x 16-thread tiles at 4096^3, where their longer
// fill and drain costs them most); the small and mid tiles and the
// partial-wave fractions in plain_select were then fitted to B200 sweeps of
// 256..16384 cubes and of 1000, 3001, 5003 and 8191: the model's pick is
// within 0.2% of the fastest measured configuration at every one of those
// sizes.  The 8-warp 128 x 64 tiles and the producer-warp tiles were measured
// later (B200, interleaved timing at 1000..8192): the 4-stage producer tile
// ties the 3-stage tile within 0.2% from 4096^3 up and is 3.4% (1024^3) to
// 5.6% (1000^3) faster when the problem is one partial wave with a lone CTA
// per SM and beta = 0; the 8-warp tiles are slower everywhere.  The model
// gives the 4-stage producer tile its measured lone-CTA throughput (1.045 of
// the 3-stage tile's) and a full-wave figure that keeps multi-wave problems
// on the tiles that measured best there: at 2048^3 its two CTAs per SM fit the
// 512 tiles in two waves, yet the 64 x 64 tile is 1.6-2.2% faster.  The
// 28 x 256 tiles were measured the same way at 768..12288.  The 4-stage one
// (one CTA per SM) is 9-11% faster than the previous pick at 1000^3 and
// 1024^3 and 8-9% at 896^3 (both betas) and slower elsewhere; 0.80
// reproduces those picks.  The 3-stage one (two CTAs per SM) is 10-12%
// faster at 2048^3, 1.4-1.9% at 3072^3 and 6144^3, within 0.5% at 4096^3,
// 8192^3 and 12288^3, 3% slower at 1280^3 and 2560^3 and far slower at
// 1536^3 (330 tiles: a third, near-empty wave); 0.99 picks it at 2048^3,
// 4096^3 and 6144^3 and leaves 8192^3 on the 128 x 64 tile, and its lone
// figure, 0.95, keeps 896..1024 on the 4-stage tile, 1-3% faster there.
// (Measured and dropped: 6 stages, 1-3% slower than 4; eight 7 x 4-thread
// warps, 2-5% slower at beta = 0; 32-row rasterisation bands, no change.)
static const ConfigDesc kConfigs[] = {
    describe<C0>("tma_128x256_w8_t8x16_s4", 0.840f),   describe<C1>("tma_128x128_w8_t8x8_s3", 0.900f),
    describe<C2>("tma_128x128_w4_t8x16_s3", 0.875f),   describe<C3>("tma_64x128_w4_t8x8_s4", 0.920f),
    describe<C4>("tma_64x64_w2_t8x8_s4", 0.700f),      describe<C5>("tma_64x128_w4_t8x8_s3", 0.994f),
    describe<C6>("tma_128x64_w4_t8x8_s3", 1.000f),     describe<S0>("tma_64x64_w4_t8x4_s4", 0.860f),
    describe<S1>("tma_32x64_w2_t8x4_s4", 0.700f),      describe<C8>("cpa_128x256_w8_t8x16_s4", 1.000f),
    describe<C9>("cpa_128x128_w8_t8x8_s3", 0.920f),    describe<C11>("cpa_64x128_w4_t8x8_s4", 0.810f),
    describe<C12>("cpa_64x64_w2_t8x8_s4", 0.630f),     describe<C14>("cpa_128x64_w4_t8x8_s3", 0.890f),
    describe<W0>("tma_128x64_w8_t8x4_s3", 0.850f),     describe<W1>("tma_128x64_w8_t8x4_s4", 0.900f),
    describe<P0>("tma_128x64_w4p_t8x8_s3", 0.900f),    describe<P1>("tma_128x64_w4p_t8x8_s4", 0.900f, 1.045f),
    describe<T0>("tma_28x256_w4p_t7x8_s4", 0.800f),    describe<T3>("tma_28x256_w4p_t7x8_s3", 0.990f, 0.950f),
};
constexpr int kNumConfigs = sizeof(kConfigs) / sizeof(kConfigs[0]);

static int occupancy(int cfg) {
    static int occ[64][kNumConfigs];
    static bool have[64][kNumConfigs];
    static std::mutex mu;
    const DeviceInfo& d = device_info();
    if (d.device < 0 || d.device >= 64) return 1;
    std::lock_guard<std::mutex> lock(mu);
    if (!have[d.device][cfg]) {
        const ConfigDesc& c = kConfigs[cfg];
        int o = 0;
        cudaFuncSetAttribute(c.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, c.smem);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, c.kernel, c.threads, c.smem) !=
                cudaSuccess ||
            o < 1)
            o = 1;
        occ[d.device][cfg] = o;
        have[d.device][cfg] = true;
    }
    return occ[d.device][cfg];
}

static bool tma_ok(const float* A, int lda, const float* B, int ldb) {
    return (lda % 4 == 0) && (ldb % 4 == 0) && (reinterpret_cast<uintptr_t>(A) % 16 == 0) &&
           (reinterpret_cast<uintptr_t>(B) % 16 == 0);
}

}  // namespace ffma

int plain_config_count() { return ffma::kNumConfigs; }
const char* plain_config_name(int cfg) {
    return (cfg >= 0 && cfg < ffma::kNumConfigs) ? ffma::kConfigs[cfg].name : nullptr;
}
int plain_config_tile(int cfg, int* bm, int* bn) {
    if (cfg < 0 || cfg >= ffma::kNumConfigs) return SGEMM_B200_ERR_INVALID_ARG;
    *bm = ffma::kConfigs[cfg].bm;
    *bn = ffma::kConfigs[cfg].bn;
    return SGEMM_B200_OK;
}

// Pick the configuration with the smallest modelled time.  A configuration
// with `occ` resident CTAs per SM runs tiles in waves of SMs x occ; one CTA of
// a full wave takes t = occ * BM * BN / efficiency (per-SM throughput shared
// by occ CTAs).  The last, partial wave leaves r = ceil(remainder / SMs) < occ
// CTAs on the busiest SM, which then runs at a fraction e(r) of its full
// throughput (fewer warps to hide latency), so that wave takes
// t * (r / occ) / e(r).  e(1) = 0.70, e(2) = e(3) = 0.90 were fitted to the
// same B200 measurements as the efficiencies.  One exception, also measured:
// when the whole problem is that one partial wave with a single CTA per SM
// and C is not read (beta == 0), e(1) = 0.82 -- the lone CTA's epilogue then
// only writes, and nothing else on the SM waits for it (1000^3 and 1024^3 at
// beta = 0 run 3.6-4.5% faster on the 128 x 64 tile than on 64 x 64, while at
// beta = 0.5 the 64 x 64 tile is 3% faster).
static double partial_wave_cost(int r, int occ, bool alone, bool reads_c) {
    if (r >= occ) return 1.0;
    const double e = r == 1 ? (alone && !reads_c ? 0.82 : 0.70) : 0.90;
    return (double(r) / occ) / e;
}

static int select_for_loader(int m, int n, int k, int loader, bool reads_c) {
    using namespace ffma;
    const DeviceInfo& d = device_info();
    const int sms = d.sm_count > 0 ? d.sm_count : 148;
    int best = -1;
    double best_t = 1e300;
    for (int c = 0; c < kNumConfigs; ++c) {
        const ConfigDesc& cd = kConfigs[c];
        if (cd.loader != loader) continue;
        const int occ = occupancy(c);
        const double tiles = double(div_up(m, cd.bm)) * div_up(n, cd.bn);
        const double slots = double(sms) * occ;
        const double full = std::floor(tiles / slots);
        const double rem = tiles - full * slots;
        double waves = full;
        const int r = rem > 0 ? static_cast<int>(std::ceil(rem / sms)) : 0;
        if (rem > 0) waves += partial_wave_cost(r, occ, full == 0, reads_c);
        // a lone CTA per SM runs one warp per scheduler: latency, not the FMA
        // pipe, limits it, and the producer-warp tile hides more of it
        const double eff = (full == 0 && r == 1 && cd.lone > 0) ? cd.lone : cd.efficiency;
        const double t = waves * occ * double(cd.bm) * cd.bn / eff;
        if (best < 0 || t < best_t * 0.999) {
            best_t = t;
            best = c;
        }
    }
    (void)k;
    return best;
}

int plain_select(int m, int n, int k, const float* A, int lda, const float* B, int ldb,
                 bool reads_c) {
    using namespace ffma;
    const int loader = (k == 0 || tma_ok(A, lda, B, ldb)) ? kLoaderTma : kLoaderAsync4;
    return select_for_loader(m, n, k, loader, reads_c);
}

namespace ffma {

// Row copy into a 16-byte-aligned pitch (the pack step for strides TMA cannot
// describe), for up to two matrices in one launch: block b copies rows b,
// b + gridDim.x, ... of A's rows followed by B's; within a row the threads
// take consecutive columns (coalesced), eight loads in flight per thread
// before their stores.  HBM-bound; the padding columns are not written (the
// TMA kernel reads only the first `cols` of each row).
struct PackJob {
    const float* src;
    float* dst;
    int rows, cols, ld_src, ld_dst;
};

constexpr int kPackThreads = 256;
constexpr int kPackUnroll = 8;

__global__ void __launch_bounds__(kPackThreads) pack_rows_kernel(const PackJob a, const PackJob b) {
    const int total = a.rows + b.rows;
    for (int r = blockIdx.x; r < total; r += gridDim.x) {
        const bool in_a = r < a.rows;
        const int row = in_a ? r : r - a.rows;
        const int cols = in_a ? a.cols : b.cols;
        const float* __restrict__ src =
            (in_a ? a.src : b.src) + (int64_t)row * (in_a ? a.ld_src : b.ld_src);
        float* __restrict__ dst =
            (in_a ? a.dst : b.dst) + (int64_t)row * (in_a ? a.ld_dst : b.ld_dst);
        for (int c0 = 0; c0 < cols; c0 += kPackUnroll * kPackThreads) {
            float v[kPackUnroll];
#pragma unroll
            for (int u = 0; u < kPackUnroll; ++u) {
                const int c = c0 + u * kPackThreads + (int)threadIdx.x;
                v[u] = c < cols ? src[c] : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < kPackUnroll; ++u) {
                const int c = c0 + u * kPackThreads + (int)threadIdx.x;
                if (c < cols) dst[c] = v[u];
            }
        }
    }
}

// Work (m*n*k) above which copying unaligned operands to aligned rows and
// running the TMA kernel beats the 4-byte cp.async loader.
constexpr double kPackMinWork = 134217728.0;  // 512^3

// Operands the plain path copies to aligned rows before its TMA kernel:
// bit 0 A, bit 1 B; 0 when the kernel reads them in place.
static int pack_mask(int m, int n, int k, const float* A, int lda, const float* B, int ldb) {
    if (k <= 0 || tma_ok(A, lda, B, ldb) || double(m) * n * k < kPackMinWork) return 0;
    const bool pa = (lda % 4 != 0) || (reinterpret_cast<uintptr_t>(A) % 16 != 0);
    const bool pb = (ldb % 4 != 0) || (reinterpret_cast<uintptr_t>(B) % 16 != 0);
    return (pa ? 1 : 0) | (pb ? 2 : 0);
}

// One launch for both operands (a job with rows == 0 is skipped): eight
// blocks per SM, each looping over rows.
static void pack(const PackJob& a, const PackJob& b, cudaStream_t s) {
    const int total = a.rows + b.rows;
    const int sms = device_info().sm_count > 0 ? device_info().sm_count : 148;
    const int grid = std::max(1, std::min(total, sms * 8));
    pack_rows_kernel<<<grid, kPackThreads, 0, s>>>(a, b);
}

}  // namespace ffma

int plain_launch(int cfg, int m, int n, int k, float alpha, const float* A, int lda,
                 const float* B, int ldb, float beta, float* C, int ldc, cudaStream_t stream) {
    return plain_launch_acc(cfg, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, nullptr, nullptr,
                            0, stream);
}

int plain_launch_acc(int cfg, int m, int n, int k, float alpha, const float* A, int lda,
                     const float* B, int ldb, float beta, float* C, int ldc, const float* acc_in,
                     float* acc_out, int ld_acc, cudaStream_t stream) {
    using namespace ffma;
    if (m == 0 || n == 0) return SGEMM_B200_OK;
    if (!device_is_sm100()) return SGEMM_B200_ERR_UNSUPPORTED;
    if ((acc_in || acc_out) &&
        (ld_acc < n || ld_acc % 4 != 0 || reinterpret_cast<uintptr_t>(acc_in) % 16 != 0 ||
         reinterpret_cast<uintptr_t>(acc_out) % 16 != 0))
        return SGEMM_B200_ERR_INVALID_ARG;
    // carried accumulators: the caller keeps its operands TMA-aligned (no pack step)
    const int mask = (cfg < 0 && !acc_in && !acc_out) ? pack_mask(m, n, k, A, lda, B, ldb) : 0;
    if (mask) {
        // Unaligned strides on a large problem: copy the offending operand(s) to
        // 16-byte-aligned rows (stream-ordered scratch from the library pool)
        // and run the TMA kernel.  Same arithmetic, same bits.
        cudaMemPool_t pool = library_pool();
        if (pool) {
            const bool pa = (mask & 1) != 0, pb = (mask & 2) != 0;
            const int lda2 = pa ? (k + 3) / 4 * 4 : lda, ldb2 = pb ? (n + 3) / 4 * 4 : ldb;
            float *A2 = nullptr, *B2 = nullptr;
            cudaError_t e = cudaSuccess;
            if (pa) e = cudaMallocFromPoolAsync(&A2, sizeof(float) * (size_t)m * lda2, pool, stream);
            if (e == cudaSuccess && pb)
                e = cudaMallocFromPoolAsync(&B2, sizeof(float) * (size_t)k * ldb2, pool, stream);
            if (e == cudaSuccess) {
                const PackJob ja = pa ? PackJob{A, A2, m, k, lda, lda2} : PackJob{};
                const PackJob jb = pb ? PackJob{B, B2, k, n, ldb, ldb2} : PackJob{};
                pack(ja, jb, stream);
                const int s = plain_launch(-1, m, n, k, alpha, pa ? A2 : A, lda2, pb ? B2 : B,
                                           ldb2, beta, C, ldc, stream);
                if (A2) cudaFreeAsync(A2, stream);
                if (B2) cudaFreeAsync(B2, stream);
                return s;
            }
            if (A2) cudaFreeAsync(A2, stream);
            if (B2) cudaFreeAsync(B2, stream);
            cudaGetLastError();  // fall through to the cp.async loader
        }
    }
    if (cfg < 0) cfg = plain_select(m, n, k, A, lda, B, ldb, beta != 0.0f);
    if (cfg >= kNumConfigs) return SGEMM_B200_ERR_INVALID_ARG;
    const ConfigDesc& cd = kConfigs[cfg];
    if (cd.loader == kLoaderTma && k > 0 && !tma_ok(A, lda, B, ldb))
        return SGEMM_B200_ERR_INVALID_ARG;

    Params p;
    p.op.m = m;
    p.op.n = n;
    p.op.k = k;
    p.op.lda = lda;
    p.op.ldb = ldb;
    p.op.ldc = ldc;
    p.op.alpha = alpha;
    p.op.beta = beta;
    p.op.A = A;
    p.op.B = B;
    p.op.C = C;
    p.op.vec_c = (ldc % 4 == 0) && (reinterpret_cast<uintptr_t>(C) % 16 == 0);
    p.status = device_status_ptr();
    if (!p.status) return SGEMM_B200_ERR_CUDA;
    p.tiles_m = div_up(m, cd.bm);
    p.tiles_n = div_up(n, cd.bn);
    p.acc_in = acc_in;
    p.acc_out = acc_out;
    p.ld_acc = ld_acc;

    CUtensorMap tmA, tmB;
    std::memset(&tmA, 0, sizeof(tmA));
    std::memset(&tmB, 0, sizeof(tmB));
    if (cd.loader == kLoaderTma && k > 0) {
        if (!encode_tensor_map_2d(&tmA, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, A, (uint64_t)k,
                                  (uint64_t)m, (uint64_t)lda * 4, 32, cd.bm,
                                  CU_TENSOR_MAP_SWIZZLE_128B) ||
            !encode_tensor_map_2d(&tmB, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, B, (uint64_t)n,
                                  (uint64_t)k, (uint64_t)ldb * 4, cd.bn, 32,
                                  CU_TENSOR_MAP_SWIZZLE_NONE))
            return SGEMM_B200_ERR_CUDA;
    }
    occupancy(cfg);  // sets the dynamic shared-memory attribute once per device
    const int grid = p.tiles_m * p.tiles_n;
    cd.kernel<<<grid, cd.threads, cd.smem, stream>>>(tmA, tmB, p);
    return cuda_status(cudaGetLastError());
}

}  // namespace sgb

// ---------------------------------------------------------------- C ABI --

extern "C" int sgemm_b200_with_config(int cfg, int m, int n, int k, const float* alpha,
                                      const float* A, int lda, const float* B, int ldb,
                                      const float* beta, float* C, int ldc,
                                      sgemm_b200_stream_t stream) {
    int s = sgb::check_gemm_args(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    if (s == SGEMM_B200_OK)
        s = sgb::plain_launch(cfg, m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc,
                              sgb::as_stream(stream));
    sgb::set_last_status(s);
    return s;
}

extern "C" int sgemm_b200(int m, int n, int k, const float* alpha, const float* A, int lda,
                          const float* B, int ldb, const float* beta, float* C, int ldc,
                          sgemm_b200_stream_t stream) {
    return sgemm_b200_with_config(-1, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream);
}

extern "C" void sgemm(int m, int n, int k, const float* alpha, float* A, int lda, float* B,
                      int ldb, const float* beta, float* C, int ldc) {
    sgemm_b200(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, nullptr);
}

extern "C" int sgemm_b200_config_count(void) { return sgb::plain_config_count(); }

extern "C" const char* sgemm_b200_config_name(int cfg) { return sgb::plain_config_name(cfg); }

extern "C" int sgemm_b200_select_config_beta(int m, int n, int k, const float* A, int lda,
                                             const float* B, int ldb, const float* beta) {
    if (m <= 0 || n <= 0 || k < 0) return -1;
    const bool reads_c = beta == nullptr || *beta != 0.0f;
    // the kernel that runs: after a pack step the operands are TMA-aligned
    if (sgb::ffma::pack_mask(m, n, k, A, lda, B, ldb))
        return sgb::select_for_loader(m, n, k, sgb::ffma::kLoaderTma, reads_c);
    return sgb::plain_select(m, n, k, A, lda, B, ldb, reads_c);
}

extern "C" int sgemm_b200_select_config(int m, int n, int k, const float* A, int lda,
                                        const float* B, int ldb, const float* C, int ldc) {
    (void)C;
    (void)ldc;
    return sgemm_b200_select_config_beta(m, n, k, A, lda, B, ldb, nullptr);
}

extern "C" int sgemm_b200_packs(int m, int n, int k, const float* A, int lda, const float* B,
                                int ldb) {
    if (m <= 0 || n <= 0 || k < 0) return 0;
    return sgb::ffma::pack_mask(m, n, k, A, lda, B, ldb);
}
