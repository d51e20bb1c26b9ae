// texld.cu — the texture-fetch loader: the plain FFMA GEMM with A and B read
// through texture objects.
//
// Replaces the reference's pre-Ampere path (src/sgemm.cuh:49-89 with
// src/kernels/128x128x8_texld.cuh): when A and B rows are 16-byte aligned
// (lda and ldb multiples of 4, A and B 16-byte aligned -- the reference's
// `is_aligned`), sgemm() there wraps A and B in linear texture objects and its
// kernel fetches them as float4 texels (tex1Dfetch<float4>); otherwise it
// falls back to the plain-load kernel.  Same here: aligned operands go through
// texld_gemm_kernel, others to sgemm_b200.  On a B200 the TMA loader is the
// fast path; this one exists so that code written against the texture path
// (or that wants A and B read through the texture cache) has it, with the
// plain path's exact arithmetic -- results equal sgemm_b200's bit for bit.
//
// Kernel: the 128 x 64 tile of the plain path (4 warps, 8 x 8 per thread,
// the same lane map, packed-FMA core and epilogue) with a two-stage
// register-staged pipeline: the next k block's texels are fetched into
// registers while the current block is computed from shared memory, then
// stored into the other stage (A into the 128-byte swizzled k-contiguous
// layout the core reads, B row by row).  Texels past k in a row of A, past n
// in a row of B, and rows past m or k are replaced by zeros, so the padded
// terms add exact +0 like the TMA loader's out-of-bounds fill.
//
// Texture objects live as long as the work that reads them: each call
// records an event after its kernel, and a reaper thread destroys the call's
// two objects once that event completes, so the call itself never waits.
#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>

#include "common.h"
#include "ffma_kernel.cuh"
#include "plain.h"

namespace sgb {
namespace texld {

using C = ffma::Cfg<128, 64, 4, 1, 8, 2, ffma::kLoaderAsync4, 2>;  // 2 stages, 48 KB
constexpr int A4 = C::BM * C::BK / 4 / C::THREADS;  // A texels per thread per stage (8)
constexpr int B4 = C::BK * C::BN / 4 / C::THREADS;  // B texels per thread per stage (4)
static_assert(A4 * C::THREADS * 4 == C::BM * C::BK && B4 * C::THREADS * 4 == C::BK * C::BN, "");

struct Params {
    ffma::Operands op;
    cudaTextureObject_t ta, tb;  // float4 texels of A and B
    int offa, offb;              // texel of A[0] / B[0] (a texture's base is aligned down)
    int tiles_m, tiles_n;
};

__device__ __forceinline__ float4 masked(float4 v, int valid) {
    // keep the first `valid` (0..4) components
    if (valid < 4) v.w = 0.0f;
    if (valid < 3) v.z = 0.0f;
    if (valid < 2) v.y = 0.0f;
    if (valid < 1) v.x = 0.0f;
    return v;
}

// Texels of k block kb: thread t takes A texels (row r, texel q of 8) for
// e = t + i*THREADS, r = e / 8, q = e % 8, and B texels (row r of 32, texel q
// of BN/4) for e = t + i*THREADS, r = e / (BN/4), q = e % (BN/4).
__device__ __forceinline__ void fetch(const Params& p, int m0, int n0, int kb, float4 (&a)[A4],
                                      float4 (&b)[B4]) {
    const int k0 = kb * C::BK;
#pragma unroll
    for (int i = 0; i < A4; ++i) {
        const int e = threadIdx.x + i * C::THREADS;
        const int r = e >> 3, q = e & 7;
        const int row = m0 + r, col = k0 + 4 * q;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (row < p.op.m && col < p.op.k)
            v = masked(tex1Dfetch<float4>(p.ta, p.offa + (int)(((int64_t)row * p.op.lda + col) >> 2)),
                       p.op.k - col);
        a[i] = v;
    }
#pragma unroll
    for (int i = 0; i < B4; ++i) {
        const int e = threadIdx.x + i * C::THREADS;
        const int r = e / (C::BN / 4), q = e % (C::BN / 4);
        const int row = k0 + r, col = n0 + 4 * q;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (row < p.op.k && col < p.op.n)
            v = masked(tex1Dfetch<float4>(p.tb, p.offb + (int)(((int64_t)row * p.op.ldb + col) >> 2)),
                       p.op.n - col);
        b[i] = v;
    }
}

__device__ __forceinline__ void store(uint8_t* st, const float4 (&a)[A4], const float4 (&b)[B4]) {
#pragma unroll
    for (int i = 0; i < A4; ++i) {
        const int e = threadIdx.x + i * C::THREADS;
        const int r = e >> 3, q = e & 7;
        // the 128-byte swizzle the TMA loader writes: 16-byte chunk q of row r
        // lands at chunk q ^ (r % 8)
        *reinterpret_cast<float4*>(st + r * 128 + ((q ^ (r & 7)) << 4)) = a[i];
    }
#pragma unroll
    for (int i = 0; i < B4; ++i) {
        const int e = threadIdx.x + i * C::THREADS;
        const int r = e / (C::BN / 4), q = e % (C::BN / 4);
        *reinterpret_cast<float4*>(st + C::A_BYTES + (r * C::BN + 4 * q) * 4) = b[i];
    }
}

__global__ void __launch_bounds__(C::THREADS, C::MINB) texld_gemm_kernel(const Params p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = align_smem_1024(smem_raw);
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int wm = warp / C::WN, wn = warp % C::WN;
    int lm, ln;
    ffma::lane_coords(lane, lm, ln);
    int tm, tn;
    ffma::tile_coords(blockIdx.x, p.tiles_m, p.tiles_n, tm, tn);
    const int m0 = tm * C::BM, n0 = tn * C::BN;
    const int nk = (p.op.k + C::BK - 1) / C::BK;
    uint32_t a_base, xa0, xa1;
    ffma::a_coords<C>(wm, lm, a_base, xa0, xa1);
    const uint32_t b_base = static_cast<uint32_t>((wn * 8 * C::TN + ln * 4) * 4);

    float acc[C::TM][C::TN];
#pragma unroll
    for (int i = 0; i < C::TM; ++i)
#pragma unroll
        for (int j = 0; j < C::TN; ++j) acc[i][j] = 0.0f;

    float4 ra[A4], rb[B4];
    if (nk > 0) {
        fetch(p, m0, n0, 0, ra, rb);
        store(smem, ra, rb);
    }
    __syncthreads();
    for (int kb = 0; kb < nk; ++kb) {
        // Stage (kb+1) % 2 was last read in iteration kb-1, which every warp
        // finished before the barrier that ended it.
        const bool more = kb + 1 < nk;
        if (more) fetch(p, m0, n0, kb + 1, ra, rb);
        const uint8_t* st = smem + (kb & 1) * C::STAGE_BYTES;
        ffma::compute_stage<C>(st, st + C::A_BYTES, a_base, xa0, xa1, b_base, acc);
        if (more) store(smem + ((kb + 1) & 1) * C::STAGE_BYTES, ra, rb);
        __syncthreads();
    }
    ffma::epilogue_any<C>(p.op, m0, n0, wm, wn, lm, ln, acc, smem);
}

// ------------------------------------------------------ texture lifetimes --

// Destroys each call's texture objects once the event recorded after its
// kernel has completed, on a thread of its own, so calls never wait.
class Reaper {
  public:
    static Reaper& get() {
        static Reaper* r = new Reaper();  // never destroyed: the thread may outlive main's statics
        return *r;
    }
    void push(int device, cudaEvent_t done, cudaTextureObject_t a, cudaTextureObject_t b) {
        std::lock_guard<std::mutex> lock(mu_);
        q_.push_back(Item{device, done, a, b});
        cv_.notify_one();
    }

  private:
    struct Item {
        int device;
        cudaEvent_t done;
        cudaTextureObject_t a, b;
    };
    Reaper() { std::thread([this] { loop(); }).detach(); }
    void loop() {
        std::unique_lock<std::mutex> lock(mu_);
        while (true) {
            cv_.wait(lock, [&] { return !q_.empty(); });
            Item it = q_.front();
            q_.pop_front();
            lock.unlock();
            cudaSetDevice(it.device);
            cudaEventSynchronize(it.done);
            cudaDestroyTextureObject(it.a);
            cudaDestroyTextureObject(it.b);
            cudaEventDestroy(it.done);
            lock.lock();
        }
    }
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Item> q_;
};

// A linear texture over [base, base + bytes) whose start is `base` aligned
// down to the device's texture alignment; *offset receives the texel index of
// `base` (which is 16-byte aligned, so it is a whole texel).
static bool make_texture(cudaTextureObject_t* t, int* offset, const float* base, size_t bytes) {
    const DeviceInfo& di = device_info();
    int align = 0;
    if (cudaDeviceGetAttribute(&align, cudaDevAttrTextureAlignment, di.device) != cudaSuccess ||
        align < 16)
        align = 512;
    const uintptr_t b = reinterpret_cast<uintptr_t>(base);
    const uintptr_t b0 = b / align * align;
    *offset = (int)((b - b0) / 16);
    cudaResourceDesc res;
    std::memset(&res, 0, sizeof(res));
    res.resType = cudaResourceTypeLinear;
    res.res.linear.devPtr = reinterpret_cast<void*>(b0);
    res.res.linear.desc = cudaCreateChannelDesc<float4>();
    res.res.linear.sizeInBytes = bytes + (b - b0);
    cudaTextureDesc td;
    std::memset(&td, 0, sizeof(td));
    td.readMode = cudaReadModeElementType;
    return cudaCreateTextureObject(t, &res, &td, nullptr) == cudaSuccess;
}

// Texels a linear texture may hold on this device.
static size_t max_texels() {
    int w = 0;
    if (cudaDeviceGetAttribute(&w, cudaDevAttrMaxTexture1DLinearWidth, device_info().device) !=
            cudaSuccess ||
        w <= 0)
        return size_t(1) << 27;
    return (size_t)w;
}

// The reference's condition for its texture path (src/sgemm.cuh:54-55).
static bool aligned(const float* A, int lda, const float* B, int ldb) {
    return (lda % 4 == 0) && (ldb % 4 == 0) && (reinterpret_cast<uintptr_t>(A) % 16 == 0) &&
           (reinterpret_cast<uintptr_t>(B) % 16 == 0);
}

static int launch(int m, int n, int k, float alpha, const float* A, int lda, const float* B,
                  int ldb, float beta, float* C_, int ldc, cudaStream_t stream) {
    if (m == 0 || n == 0) return SGEMM_B200_OK;
    if (!device_is_sm100()) return SGEMM_B200_ERR_UNSUPPORTED;
    if (k == 0 || !aligned(A, lda, B, ldb))  // as the reference: the plain-load kernel
        return plain_launch(-1, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc, stream);
    // Operands larger than a linear texture may hold (or than 32-bit texel
    // indices reach) take the plain-load kernel too.
    const size_t a_bytes = ((size_t)(m - 1) * lda + k) * sizeof(float);
    const size_t b_bytes = ((size_t)(k - 1) * ldb + n) * sizeof(float);
    const size_t limit = std::min(max_texels(), size_t(1) << 30) - 64;  // room for the offset
    if ((a_bytes + 15) / 16 > limit || (b_bytes + 15) / 16 > limit)
        return plain_launch(-1, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc, stream);
    cudaTextureObject_t ta = 0, tb = 0;
    int offa = 0, offb = 0;
    // round the extents up to whole texels (the last texel of a row may run past k or n)
    if (!make_texture(&ta, &offa, A, (a_bytes + 15) / 16 * 16)) return SGEMM_B200_ERR_CUDA;
    if (!make_texture(&tb, &offb, B, (b_bytes + 15) / 16 * 16)) {
        cudaDestroyTextureObject(ta);
        return SGEMM_B200_ERR_CUDA;
    }
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
    p.op.C = C_;
    p.op.vec_c = (ldc % 4 == 0) && (reinterpret_cast<uintptr_t>(C_) % 16 == 0);
    p.ta = ta;
    p.tb = tb;
    p.offa = offa;
    p.offb = offb;
    p.tiles_m = div_up(m, C::BM);
    p.tiles_n = div_up(n, C::BN);
    static std::once_flag attr[64];
    const int dev = device_info().device;
    if (dev < 0 || dev >= 64) return SGEMM_B200_ERR_CUDA;
    std::call_once(attr[dev], [] {
        cudaFuncSetAttribute(texld_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             C::SMEM_BYTES);
    });
    texld_gemm_kernel<<<p.tiles_m * p.tiles_n, C::THREADS, C::SMEM_BYTES, stream>>>(p);
    int st = cuda_status(cudaGetLastError());
    cudaEvent_t done = nullptr;
    if (cudaEventCreateWithFlags(&done, cudaEventDisableTiming) == cudaSuccess &&
        cudaEventRecord(done, stream) == cudaSuccess) {
        Reaper::get().push(dev, done, ta, tb);
    } else {
        // cannot track the kernel: wait for it before the objects go
        if (done) cudaEventDestroy(done);
        cudaStreamSynchronize(stream);
        cudaDestroyTextureObject(ta);
        cudaDestroyTextureObject(tb);
        if (st == SGEMM_B200_OK) st = SGEMM_B200_ERR_CUDA;
    }
    return st;
}

}  // namespace texld
}  // namespace sgb

extern "C" int sgemm_b200_texld(int m, int n, int k, const float* alpha, const float* A, int lda,
                                const float* B, int ldb, const float* beta, float* C, int ldc,
                                sgemm_b200_stream_t stream) {
    int s = sgb::check_gemm_args(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    if (s == SGEMM_B200_OK)
        s = sgb::texld::launch(m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc,
                               sgb::as_stream(stream));
    sgb::set_last_status(s);
    return s;
}
