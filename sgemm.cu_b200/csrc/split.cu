// split.cu — split-precision FP32 GEMM on the 5th-generation tensor cores.
//
// No reference counterpart: the reference has no tensor-core path at all
// (src/kernels/*.cuh are FFMA only).  The contract is the reference sgemm()'s
// (src/sgemm.cuh:19-30): C := alpha*A*B + beta*C, FP32 row-major, beta == 0
// never reads C.
//
// BF16X6: every FP32 operand x is split exactly into three BF16 terms
//   x_h = bf16(x), x_m = bf16(x - x_h), x_l = bf16(x - x_h - x_m)
// and A*B is formed from the six cross products that carry the FP32 bits:
//   hh + (hm + mh + hl + lh + mm)       (ml, lm, ll are below 2^-24 |a||b|).
// TF32X3: x_h = tf32(x), x_l = tf32(x - x_h);  A*B = hh + (hl + lh).
//
// The products run as tcgen05.mma (kind::f16 with BF16 inputs, or
// kind::tf32) with FP32 accumulation in tensor memory.  Accuracy:
//  - the dominant hh term (D1) and the correction terms (D2) accumulate in
//    separate TMEM accumulators;
//  - D1 only ever accumulates one K chunk (KCHUNK) in the tensor core: eight
//    drain warps then add the chunk into FP32 registers with round-to-nearest
//    before the next chunk overwrites D1.  Long accumulations inside the
//    tensor core lose accuracy with K; chunk sums added on the CUDA cores do
//    not.  D2 is ~2^-8 of D1, so its own accumulation error is negligible and
//    it is read once, at the end;
//  - every k step issues its correction MMAs before its hh MMA, so while the
//    drain warps empty D1 the tensor core still has the next step's
//    corrections to work on.
//
// Kernel shape: one CTA of 10 warps per 128 x 256 output tile.
//   warps 0..7  drain + epilogue: warp w reads TMEM lanes 32*(w%4).. (rows)
//               and columns 128*(w/4)..+127, keeps 128 FP32 running sums,
//               and finally adds D2, applies alpha/beta and stores float4s
//   warp 8      TMA producer (one lane): one 3-D box per operand per stage
//               brings every split plane of a 64-byte K slice (64-byte swizzle)
//   warp 9      MMA issuer (one lane): tcgen05.mma M=128 N=256
// TMEM (512 columns): D1 at 0, D2 at 256.
// Every mbarrier wait is bounded (ptx.cuh); on expiry the status word is
// set, in-flight copies are drained with bounded waits and TMEM is freed.
//
// A split pre-pass writes the operand planes (A as [split][M][Kp], B
// transposed to [split][N][Kp], both K-major) into a workspace.
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.h"
#include "plain.h"
#include "ptx.cuh"
#include "split.h"

namespace sgb {
namespace split {

constexpr int BM = 128, BN = 256;
constexpr int DRAIN_WARPS = 8, PRODUCER_WARP = 8, MMA_WARP = 9;
constexpr int THREADS = 32 * (DRAIN_WARPS + 2);
constexpr int TMEM_COLS = 512;
constexpr int KCHUNK = 256;  // K depth D1 accumulates in the tensor core before a drain

template <int PATH>
struct Traits;

template <>
struct Traits<SGEMM_B200_PATH_BF16X6> {
    static constexpr int NSPLIT = 3, ESZ = 2, BK = 32, KMMA = 16, STAGES = 3;
    static constexpr uint32_t FMT = 1;  // BF16
    static constexpr int NPROD = 6;
    // (a split, b split) in issue order: the corrections (D2) first, hh (D1) last
    __device__ static constexpr int pa(int i) {
        return i == 0 ? 0 : i == 1 ? 1 : i == 2 ? 0 : i == 3 ? 2 : i == 4 ? 1 : 0;
    }
    __device__ static constexpr int pb(int i) {
        return i == 0 ? 1 : i == 1 ? 0 : i == 2 ? 2 : i == 3 ? 0 : i == 4 ? 1 : 0;
    }
};

template <>
struct Traits<SGEMM_B200_PATH_TF32X3> {
    static constexpr int NSPLIT = 2, ESZ = 4, BK = 16, KMMA = 8, STAGES = 4;
    static constexpr uint32_t FMT = 2;  // TF32
    static constexpr int NPROD = 3;
    __device__ static constexpr int pa(int i) { return i == 1 ? 1 : 0; }
    __device__ static constexpr int pb(int i) { return i == 0 ? 1 : 0; }
};

template <int PATH>
struct Layout {
    using T = Traits<PATH>;
    static constexpr int ROW_BYTES = T::BK * T::ESZ;  // 64: one swizzle-64 row
    static_assert(ROW_BYTES == 64, "64-byte K rows");
    static constexpr int A_PLANE = BM * ROW_BYTES;    // 8 KB
    static constexpr int B_PLANE = BN * ROW_BYTES;    // 16 KB
    static constexpr int A_BYTES = T::NSPLIT * A_PLANE;
    static constexpr int B_BYTES = T::NSPLIT * B_PLANE;
    static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
    static constexpr int SMEM_BYTES = T::STAGES * STAGE_BYTES + 1024;
    static constexpr int STEPS = T::BK / T::KMMA;           // MMA k steps per stage
    static constexpr int CHUNK_STEPS = KCHUNK / T::KMMA;    // k steps per D1 chunk
    static_assert(KCHUNK % T::BK == 0, "whole stages per chunk");
    static_assert(SMEM_BYTES <= 227 * 1024, "shared memory budget");
};

struct Params {
    int m, n, k;
    int ldc;
    float alpha, beta;
    float* C;
    int* status;
    int tiles_m, tiles_n;
    int vec_c;
};

__device__ __forceinline__ void tile_coords(int bid, int tiles_m, int tiles_n, int& tm, int& tn) {
    constexpr int G = 8;
    const int per_group = G * tiles_n;
    const int gid = bid / per_group;
    const int first = gid * G;
    const int gsz = min(tiles_m - first, G);
    const int r = bid % per_group;
    tm = first + r % gsz;
    tn = r / gsz;
}

template <int PATH>
__global__ void __launch_bounds__(THREADS, 1)
    split_gemm_kernel(const __grid_constant__ CUtensorMap tmA,
                      const __grid_constant__ CUtensorMap tmB, const Params p) {
    using T = Traits<PATH>;
    using L = Layout<PATH>;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[T::STAGES];
    __shared__ __align__(8) uint64_t empty_bar[T::STAGES];
    __shared__ __align__(8) uint64_t d1_full_bar;
    __shared__ __align__(8) uint64_t d1_empty_bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;
    __shared__ int consumed_s;
    uint8_t* smem = align_smem_1024(smem_raw);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    int tm, tn;
    tile_coords(blockIdx.x, p.tiles_m, p.tiles_n, tm, tn);
    const int m0 = tm * BM, n0 = tn * BN;
    const int nk = (p.k + T::BK - 1) / T::BK;
    const int nsteps = nk * L::STEPS;
    const int nchunks = (nsteps + L::CHUNK_STEPS - 1) / L::CHUNK_STEPS;

    if (tid == 0) {
        for (int s = 0; s < T::STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        mbar_init(&d1_full_bar, 1);
        mbar_init(&d1_empty_bar, DRAIN_WARPS);
        abort_s = 0;
        consumed_s = 0;
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc(&tmem_base_s, TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;

    int issued = 0;
    if (warp == PRODUCER_WARP) {
        if (lane == 0) {
            // ------------------------------------------------ TMA producer --
            tma_prefetch_desc(&tmA);
            tma_prefetch_desc(&tmB);
            for (int kb = 0; kb < nk; ++kb) {
                const int s = kb % T::STAGES;
                if (kb >= T::STAGES) {
                    if (!mbar_wait(&empty_bar[s], ((kb / T::STAGES) - 1) & 1) || abort_s) {
                        abort_s = 1;
                        atomicExch(p.status, SGEMM_B200_ERR_TIMEOUT);
                        break;
                    }
                }
                uint8_t* st = smem + s * L::STAGE_BYTES;
                mbar_arrive_expect_tx(&full_bar[s], L::STAGE_BYTES);
                tma_load_3d(st, &tmA, &full_bar[s], kb * T::BK, m0, 0);
                tma_load_3d(st + L::A_BYTES, &tmB, &full_bar[s], kb * T::BK, n0, 0);
                ++issued;
            }
        }
    } else if (warp == MMA_WARP) {
        if (lane == 0) {
            // -------------------------------------------------- MMA issuer --
            constexpr uint32_t idesc = make_idesc(T::FMT, BM, BN);
            const uint32_t d1 = tmem, d2 = tmem + static_cast<uint32_t>(BN);
            int kb = 0;
            bool ok = true;
            for (; kb < nk && ok; ++kb) {
                const int s = kb % T::STAGES;
                if (!mbar_wait(&full_bar[s], (kb / T::STAGES) & 1) || abort_s) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t a0 = smem_u32(smem + s * L::STAGE_BYTES);
                const uint32_t b0 = a0 + L::A_BYTES;
#pragma unroll
                for (int j = 0; j < L::STEPS; ++j) {
                    const int step = kb * L::STEPS + j;
                    const uint32_t koff = j * T::KMMA * T::ESZ;  // 32 B per MMA K slice
                    // corrections into D2 (accumulated over the whole K)
#pragma unroll
                    for (int i = 0; i < T::NPROD - 1; ++i) {
                        const uint64_t ad = sw64_kmajor_desc(a0 + T::pa(i) * L::A_PLANE + koff);
                        const uint64_t bd = sw64_kmajor_desc(b0 + T::pb(i) * L::B_PLANE + koff);
                        const uint32_t accum = (step > 0 || i > 0) ? 1u : 0u;
                        if constexpr (T::FMT == 1)
                            mma_bf16_ss(d2, ad, bd, idesc, accum);
                        else
                            mma_tf32_ss(d2, ad, bd, idesc, accum);
                    }
                    // hh into D1, which restarts every chunk once the drain emptied it
                    const int c = step / L::CHUNK_STEPS;
                    const bool chunk_start = step % L::CHUNK_STEPS == 0;
                    if (chunk_start && c > 0) {
                        if (!mbar_wait(&d1_empty_bar, (c - 1) & 1) || abort_s) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                    }
                    {
                        const int i = T::NPROD - 1;
                        const uint64_t ad = sw64_kmajor_desc(a0 + T::pa(i) * L::A_PLANE + koff);
                        const uint64_t bd = sw64_kmajor_desc(b0 + T::pb(i) * L::B_PLANE + koff);
                        if constexpr (T::FMT == 1)
                            mma_bf16_ss(d1, ad, bd, idesc, chunk_start ? 0u : 1u);
                        else
                            mma_tf32_ss(d1, ad, bd, idesc, chunk_start ? 0u : 1u);
                    }
                    if ((step + 1) % L::CHUNK_STEPS == 0 || step + 1 == nsteps)
                        mma_commit(&d1_full_bar);  // chunk c of D1 (and all MMAs before it) done
                }
                if (!ok) break;
                mma_commit(&empty_bar[s]);  // frees the stage once these MMAs read it
            }
            if (!ok) {
                abort_s = 1;
                atomicExch(p.status, SGEMM_B200_ERR_TIMEOUT);
            }
            consumed_s = kb;
        }
    } else {
        // ------------------------------------------------ drain + epilogue --
        const int q = warp & 3, h = warp >> 2;
        const uint32_t trow = tmem + (static_cast<uint32_t>(q * 32) << 16) + h * 128;
        float acc[128];
#pragma unroll
        for (int j = 0; j < 128; ++j) acc[j] = 0.0f;
        bool ok = true;
        for (int c = 0; c < nchunks; ++c) {
            if (!mbar_wait(&d1_full_bar, c & 1) || abort_s) {
                ok = false;
                break;
            }
            tc_fence_after();
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                uint32_t r[32];
                tmem_ld_32x32b_x32(trow + g * 32, r);
                tmem_ld_wait();
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    acc[g * 32 + j] = __fadd_rn(acc[g * 32 + j], __uint_as_float(r[j]));
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&d1_empty_bar);
        }
        if (!ok) {
            abort_s = 1;
            atomicExch(p.status, SGEMM_B200_ERR_TIMEOUT);
        } else if (!abort_s) {
            // D2 is complete: the last D1 commit came after every MMA.
            const int row = m0 + q * 32 + lane;
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                uint32_t r[32];
                tmem_ld_32x32b_x32(trow + BN + g * 32, r);
                tmem_ld_wait();
                const int col0 = n0 + h * 128 + g * 32;
                if (row < p.m && col0 < p.n) {
                    float* crow = p.C + (int64_t)row * p.ldc + col0;
                    float v[32];
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        v[j] = __fmul_rn(__fadd_rn(acc[g * 32 + j], __uint_as_float(r[j])),
                                         p.alpha);
                    if (p.vec_c && col0 + 31 < p.n) {
#pragma unroll
                        for (int t = 0; t < 8; ++t) {
                            float4 o = make_float4(v[4 * t], v[4 * t + 1], v[4 * t + 2],
                                                   v[4 * t + 3]);
                            float4* dst = reinterpret_cast<float4*>(crow + 4 * t);
                            if (p.beta != 0.0f) {
                                const float4 old = *dst;
                                o.x = fmaf(old.x, p.beta, o.x);
                                o.y = fmaf(old.y, p.beta, o.y);
                                o.z = fmaf(old.z, p.beta, o.z);
                                o.w = fmaf(old.w, p.beta, o.w);
                            }
                            *dst = o;
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            if (col0 + j < p.n) {
                                float o = v[j];
                                if (p.beta != 0.0f) o = fmaf(crow[j], p.beta, o);
                                crow[j] = o;
                            }
                        }
                    }
                }
            }
        }
    }

    // ------------------------------------------------------------ teardown --
    tc_fence_before();
    __syncthreads();  // every TMEM load and MMA is done; consumed_s is visible
    if (warp == PRODUCER_WARP && lane == 0) {
        // Copies the MMA issuer never consumed (only after an abort) must land
        // before this CTA's shared memory is released.
        for (int j = consumed_s; j < issued; ++j)
            if (!mbar_wait(&full_bar[j % T::STAGES], (j / T::STAGES) & 1)) break;
    }
    if (warp == 0) {
        __syncwarp();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

// ------------------------------------------------------------ split pre-pass --

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

template <int PATH>
__device__ __forceinline__ void split_value(float x, float (&out)[3]) {
    if constexpr (PATH == SGEMM_B200_PATH_BF16X6) {
        const float h = __bfloat162float(__float2bfloat16_rn(x));
        const float r1 = __fsub_rn(x, h);
        const float mm = __bfloat162float(__float2bfloat16_rn(r1));
        const float r2 = __fsub_rn(r1, mm);
        out[0] = h;
        out[1] = mm;
        out[2] = __bfloat162float(__float2bfloat16_rn(r2));
    } else {
        const float h = tf32_rna(x);
        out[0] = h;
        out[1] = tf32_rna(__fsub_rn(x, h));
        out[2] = 0.0f;
    }
}

// Store 8 consecutive split values (one per plane) as 16-byte vectors.
template <int PATH>
__device__ __forceinline__ void store8(uint8_t* plane0, int64_t plane_bytes, int64_t elem,
                                       const float (&v)[8][3]) {
    using T = Traits<PATH>;
#pragma unroll
    for (int s = 0; s < T::NSPLIT; ++s) {
        uint8_t* dst = plane0 + s * plane_bytes + elem * T::ESZ;
        if constexpr (T::ESZ == 2) {
            uint32_t w[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * q][s], v[2 * q + 1][s]);
                w[q] = *reinterpret_cast<const uint32_t*>(&b2);
            }
            *reinterpret_cast<uint4*>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
        } else {
            reinterpret_cast<float4*>(dst)[0] = make_float4(v[0][s], v[1][s], v[2][s], v[3][s]);
            reinterpret_cast<float4*>(dst)[1] = make_float4(v[4][s], v[5][s], v[6][s], v[7][s]);
        }
    }
}

// A [m x lda] -> planes [split][m][kp], zero in columns k..kp-1: chunk i of
// the m * kp/8 chunks is 8 consecutive k of one row.
template <int PATH>
__device__ __forceinline__ void split_a_chunk(const float* __restrict__ A, int m, int k, int lda,
                                              int kp, uint8_t* __restrict__ out, int64_t i) {
    using T = Traits<PATH>;
    const int64_t plane_bytes = (int64_t)m * kp * T::ESZ;
    const int chunks = kp / 8;
    const int64_t r = i / chunks;
    const int c0 = (int)(i % chunks) * 8;
    float v[8][3];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float x = c0 + j < k ? A[r * lda + c0 + j] : 0.0f;
        split_value<PATH>(x, v[j]);
    }
    store8<PATH>(out, plane_bytes, r * kp + c0, v);
}

template <int PATH>
__global__ void split_a_kernel(const float* __restrict__ A, int m, int k, int lda, int kp,
                               uint8_t* __restrict__ out) {
    const int64_t total = (int64_t)m * (kp / 8);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x)
        split_a_chunk<PATH>(A, m, k, lda, kp, out, i);
}

// B [k x ldb] -> transposed planes [split][n][kp]: one 64 (k) x 64 (n) tile
// (bx along n, by along k) through shared memory, by a block of 256 threads.
template <int PATH>
__device__ __forceinline__ void split_bt_tile(const float* __restrict__ B, int k, int n, int ldb,
                                              int kp, uint8_t* __restrict__ out, int bx, int by,
                                              float (&tile)[64][65]) {
    using T = Traits<PATH>;
    const int k0 = by * 64, n0 = bx * 64;
    const int tx = threadIdx.x % 64, ty = threadIdx.x / 64;  // 256 threads
#pragma unroll 4
    for (int i = 0; i < 16; ++i) {
        const int kk = i * 4 + ty;
        const int gk = k0 + kk, gn = n0 + tx;
        tile[kk][tx] = (gk < k && gn < n) ? B[(int64_t)gk * ldb + gn] : 0.0f;
    }
    __syncthreads();
    const int64_t plane_bytes = (int64_t)n * kp * T::ESZ;
    // thread -> (row nn of B^T, 8-wide k chunk kc); 64 rows x 8 chunks = 512 items
    for (int item = threadIdx.x; item < 512; item += 256) {
        const int nn = item / 8, kc = (item % 8) * 8;
        const int gn = n0 + nn, gk = k0 + kc;
        if (gn >= n || gk >= kp) continue;
        float v[8][3];
#pragma unroll
        for (int j = 0; j < 8; ++j) split_value<PATH>(tile[kc + j][nn], v[j]);
        store8<PATH>(out, plane_bytes, (int64_t)gn * kp + gk, v);
    }
}

// Blocks loop over the 64 x 64 tiles (about 8 per SM in all) rather than one
// short block per tile.
template <int PATH>
__global__ void split_bt_kernel(const float* __restrict__ B, int k, int n, int ldb, int kp,
                                uint8_t* __restrict__ out, int tiles_n, int tiles) {
    __shared__ float tile[64][65];
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        split_bt_tile<PATH>(B, k, n, ldb, kp, out, t % tiles_n, t / tiles_n, tile);
        __syncthreads();  // the next tile's loads overwrite `tile`
    }
}

template <int PATH>
static size_t workspace_bytes(int m, int n, int k, size_t* a_bytes_out = nullptr) {
    using T = Traits<PATH>;
    const int64_t kp = ((int64_t)k + 7) / 8 * 8;
    const size_t a = (size_t)T::NSPLIT * m * kp * T::ESZ;
    const size_t b = (size_t)T::NSPLIT * n * kp * T::ESZ;
    const size_t a_al = (a + 1023) / 1024 * 1024;
    if (a_bytes_out) *a_bytes_out = a_al;
    return a_al + b + 1024;  // + alignment slack for the base
}

template <int PATH>
static int launch(int m, int n, int k, float alpha, const float* A, int lda, const float* B,
                  int ldb, float beta, float* C, int ldc, void* ws, size_t ws_bytes,
                  cudaStream_t stream) {
    using T = Traits<PATH>;
    using L = Layout<PATH>;
    size_t a_bytes = 0;
    const size_t need = workspace_bytes<PATH>(m, n, k, &a_bytes);
    if (ws_bytes < need) return SGEMM_B200_ERR_NO_MEMORY;
    uint8_t* base = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(ws) + 1023) & ~static_cast<uintptr_t>(1023));
    uint8_t* wa = base;
    uint8_t* wb = base + a_bytes;
    const int kp = (k + 7) / 8 * 8;

    {
        const int64_t total = (int64_t)m * (kp / 8);
        int64_t blocks = (total + 255) / 256;
        if (blocks > 148 * 32) blocks = 148 * 32;
        split_a_kernel<PATH><<<(int)blocks, 256, 0, stream>>>(A, m, k, lda, kp, wa);
        const int tiles_n = div_up(n, 64), tiles = tiles_n * div_up(kp, 64);
        const int sms = device_info().sm_count > 0 ? device_info().sm_count : 148;
        split_bt_kernel<PATH><<<std::min(tiles, sms * 8), 256, 0, stream>>>(B, k, n, ldb, kp, wb,
                                                                             tiles_n, tiles);
    }

    const CUtensorMapDataType dt =
        T::ESZ == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    CUtensorMap tmA, tmB;
    std::memset(&tmA, 0, sizeof(tmA));
    std::memset(&tmB, 0, sizeof(tmB));
    const uint64_t row = (uint64_t)kp * T::ESZ;
    if (!encode_tensor_map_3d(&tmA, dt, wa, (uint64_t)k, (uint64_t)m, T::NSPLIT, row,
                              row * (uint64_t)m, T::BK, BM, T::NSPLIT,
                              CU_TENSOR_MAP_SWIZZLE_64B) ||
        !encode_tensor_map_3d(&tmB, dt, wb, (uint64_t)k, (uint64_t)n, T::NSPLIT, row,
                              row * (uint64_t)n, T::BK, BN, T::NSPLIT,
                              CU_TENSOR_MAP_SWIZZLE_64B))
        return SGEMM_B200_ERR_CUDA;

    Params p;
    p.m = m;
    p.n = n;
    p.k = k;
    p.ldc = ldc;
    p.alpha = alpha;
    p.beta = beta;
    p.C = C;
    p.status = device_status_ptr();
    if (!p.status) return SGEMM_B200_ERR_CUDA;
    p.tiles_m = div_up(m, BM);
    p.tiles_n = div_up(n, BN);
    p.vec_c = (ldc % 4 == 0) && (reinterpret_cast<uintptr_t>(C) % 16 == 0);

    // The kernel's shared-memory attribute, once per device; a thread that
    // sees the flag also sees the attribute set.
    static std::atomic<bool> attr_set[64];
    static std::mutex attr_mu;
    const int dev = device_info().device;
    if (dev < 0 || dev >= 64) return SGEMM_B200_ERR_CUDA;
    if (!attr_set[dev].load(std::memory_order_acquire)) {
        std::lock_guard<std::mutex> lock(attr_mu);
        if (!attr_set[dev].load(std::memory_order_relaxed)) {
            const cudaError_t e = cudaFuncSetAttribute(
                split_gemm_kernel<PATH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                L::SMEM_BYTES);
            if (e != cudaSuccess) return cuda_status(e);
            attr_set[dev].store(true, std::memory_order_release);
        }
    }
    split_gemm_kernel<PATH><<<p.tiles_m * p.tiles_n, THREADS, L::SMEM_BYTES, stream>>>(tmA, tmB,
                                                                                      p);
    return cuda_status(cudaGetLastError());
}

// ------------------------------------------------------- grouped split GEMM --
//
// Many split-precision problems in two launches: one pre-pass that writes
// every problem's planes, and one persistent tcgen05 kernel over the tiles of
// all problems.  Per problem: two tensor maps (A planes, B planes) in global
// memory, and its own epilogue scalars.  Each tile is computed exactly as
// split_gemm_kernel computes it (same planes, same MMA order, same K chunks of
// D1, same epilogue), so every problem's result equals sgemm_b200_split's bit
// for bit, whatever else is in the launch.
//
// Persistent schedule: CTA c of G takes, in round r, the tile at position
// r*G + c (r even) or r*G + G-1-c (r odd) of a list sorted longest first (the
// snake order pairs long and short tiles).  Every role of the CTA walks the
// same sequence, so no tile index needs to pass between warps.  Across tiles
// the roles keep running counts (k blocks through the stage ring, D1 chunks)
// for mbarrier phases, and one more barrier, d2_empty, lets the MMA warp
// overwrite D2 for the next tile only after the drain warps have read it.

struct GSProblem {
    int m, n, k, ldc;
    float alpha, beta;
    float* C;
    int vec_c, pad;
};

struct GSTile {
    int prob, tm, tn, nk;
};

struct GSParams {
    const GSProblem* probs;
    const GSTile* tiles;
    const CUtensorMap* maps;  // 2 per problem: A planes, B planes
    int* status;
    int n_tiles;
};

__device__ __forceinline__ int snake_tile(int c, int r, int G) {
    return r * G + ((r & 1) ? (G - 1 - c) : c);
}

template <int PATH>
__global__ void __launch_bounds__(THREADS, 1) split_grouped_kernel(const GSParams gp) {
    using T = Traits<PATH>;
    using L = Layout<PATH>;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[T::STAGES];
    __shared__ __align__(8) uint64_t empty_bar[T::STAGES];
    __shared__ __align__(8) uint64_t d1_full_bar;
    __shared__ __align__(8) uint64_t d1_empty_bar;
    __shared__ __align__(8) uint64_t d2_empty_bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;
    __shared__ uint32_t consumed_s;
    uint8_t* smem = align_smem_1024(smem_raw);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int G = gridDim.x, cta = blockIdx.x;

    if (tid == 0) {
        for (int s = 0; s < T::STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        mbar_init(&d1_full_bar, 1);
        mbar_init(&d1_empty_bar, DRAIN_WARPS);
        mbar_init(&d2_empty_bar, DRAIN_WARPS);
        abort_s = 0;
        consumed_s = 0;
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc(&tmem_base_s, TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;

    uint32_t issued = 0;
    if (warp == PRODUCER_WARP) {
        if (lane == 0) {
            // ------------------------------------------------ TMA producer --
            uint32_t g = 0;  // k blocks issued through the stage ring
            bool ok = true;
            for (int r = 0; ok && r * G < gp.n_tiles; ++r) {
                const int t = snake_tile(cta, r, G);
                if (t >= gp.n_tiles) continue;
                const GSTile tl = gp.tiles[t];
                const CUtensorMap* tmA = gp.maps + 2 * tl.prob;
                const CUtensorMap* tmB = tmA + 1;
                tma_prefetch_desc(tmA);
                tma_prefetch_desc(tmB);
                for (int kb = 0; kb < tl.nk; ++kb, ++g) {
                    const int s = g % T::STAGES;
                    if (g >= (uint32_t)T::STAGES) {
                        if (!mbar_wait(&empty_bar[s], ((g / T::STAGES) - 1) & 1) || abort_s) {
                            abort_s = 1;
                            atomicExch(gp.status, SGEMM_B200_ERR_TIMEOUT);
                            ok = false;
                            break;
                        }
                    }
                    uint8_t* st = smem + s * L::STAGE_BYTES;
                    mbar_arrive_expect_tx(&full_bar[s], L::STAGE_BYTES);
                    tma_load_3d(st, tmA, &full_bar[s], kb * T::BK, tl.tm * BM, 0);
                    tma_load_3d(st + L::A_BYTES, tmB, &full_bar[s], kb * T::BK, tl.tn * BN, 0);
                    ++issued;
                }
            }
        }
    } else if (warp == MMA_WARP) {
        if (lane == 0) {
            // -------------------------------------------------- MMA issuer --
            constexpr uint32_t idesc = make_idesc(T::FMT, BM, BN);
            const uint32_t d1 = tmem, d2 = tmem + static_cast<uint32_t>(BN);
            uint32_t g = 0;   // k blocks consumed
            uint32_t cg = 0;  // D1 chunks committed
            int it = 0;       // tiles begun by this CTA
            bool ok = true;
            for (int r = 0; ok && r * G < gp.n_tiles; ++r) {
                const int t = snake_tile(cta, r, G);
                if (t >= gp.n_tiles) continue;
                const GSTile tl = gp.tiles[t];
                const int nsteps = tl.nk * L::STEPS;
                if (it > 0) {  // D2 of the previous tile must be read before it is reset
                    if (!mbar_wait(&d2_empty_bar, (it - 1) & 1) || abort_s) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                }
                for (int kb = 0; kb < tl.nk; ++kb, ++g) {
                    const int s = g % T::STAGES;
                    if (!mbar_wait(&full_bar[s], (g / T::STAGES) & 1) || abort_s) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a0 = smem_u32(smem + s * L::STAGE_BYTES);
                    const uint32_t b0 = a0 + L::A_BYTES;
#pragma unroll
                    for (int j = 0; j < L::STEPS; ++j) {
                        const int step = kb * L::STEPS + j;
                        const uint32_t koff = j * T::KMMA * T::ESZ;
#pragma unroll
                        for (int i = 0; i < T::NPROD - 1; ++i) {
                            const uint64_t ad =
                                sw64_kmajor_desc(a0 + T::pa(i) * L::A_PLANE + koff);
                            const uint64_t bd =
                                sw64_kmajor_desc(b0 + T::pb(i) * L::B_PLANE + koff);
                            const uint32_t accum = (step > 0 || i > 0) ? 1u : 0u;
                            if constexpr (T::FMT == 1)
                                mma_bf16_ss(d2, ad, bd, idesc, accum);
                            else
                                mma_tf32_ss(d2, ad, bd, idesc, accum);
                        }
                        const bool chunk_start = step % L::CHUNK_STEPS == 0;
                        if (chunk_start && cg > 0) {
                            if (!mbar_wait(&d1_empty_bar, (cg - 1) & 1) || abort_s) {
                                ok = false;
                                break;
                            }
                            tc_fence_after();
                        }
                        {
                            const int i = T::NPROD - 1;
                            const uint64_t ad =
                                sw64_kmajor_desc(a0 + T::pa(i) * L::A_PLANE + koff);
                            const uint64_t bd =
                                sw64_kmajor_desc(b0 + T::pb(i) * L::B_PLANE + koff);
                            if constexpr (T::FMT == 1)
                                mma_bf16_ss(d1, ad, bd, idesc, chunk_start ? 0u : 1u);
                            else
                                mma_tf32_ss(d1, ad, bd, idesc, chunk_start ? 0u : 1u);
                        }
                        if ((step + 1) % L::CHUNK_STEPS == 0 || step + 1 == nsteps) {
                            mma_commit(&d1_full_bar);
                            ++cg;
                        }
                    }
                    if (!ok) break;
                    mma_commit(&empty_bar[s]);
                }
                ++it;
            }
            if (!ok) {
                abort_s = 1;
                atomicExch(gp.status, SGEMM_B200_ERR_TIMEOUT);
            }
            consumed_s = g;
        }
    } else {
        // ------------------------------------------------ drain + epilogue --
        const int q = warp & 3, h = warp >> 2;
        const uint32_t trow = tmem + (static_cast<uint32_t>(q * 32) << 16) + h * 128;
        uint32_t cg = 0;
        int it = 0;
        bool ok = true;
        for (int r = 0; ok && r * G < gp.n_tiles; ++r) {
            const int t = snake_tile(cta, r, G);
            if (t >= gp.n_tiles) continue;
            const GSTile tl = gp.tiles[t];
            const int nchunks = (tl.nk * L::STEPS + L::CHUNK_STEPS - 1) / L::CHUNK_STEPS;
            float acc[128];
#pragma unroll
            for (int j = 0; j < 128; ++j) acc[j] = 0.0f;
            for (int c = 0; c < nchunks; ++c, ++cg) {
                if (!mbar_wait(&d1_full_bar, cg & 1) || abort_s) {
                    ok = false;
                    break;
                }
                tc_fence_after();
#pragma unroll
                for (int gq = 0; gq < 4; ++gq) {
                    uint32_t rr[32];
                    tmem_ld_32x32b_x32(trow + gq * 32, rr);
                    tmem_ld_wait();
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        acc[gq * 32 + j] = __fadd_rn(acc[gq * 32 + j], __uint_as_float(rr[j]));
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&d1_empty_bar);
            }
            if (!ok || abort_s) break;
            // D2 is complete (the tile's last D1 commit came after its MMAs):
            // read it all, release it to the MMA warp, then store C.  The
            // outputs replace the running sums in place (acc doubles as v).
            float(&v)[128] = acc;
            const float alpha = gp.probs[tl.prob].alpha;
#pragma unroll
            for (int gq = 0; gq < 4; ++gq) {
                uint32_t rr[32];
                tmem_ld_32x32b_x32(trow + BN + gq * 32, rr);
                tmem_ld_wait();
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    v[gq * 32 + j] =
                        __fmul_rn(__fadd_rn(acc[gq * 32 + j], __uint_as_float(rr[j])), alpha);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&d2_empty_bar);
            const GSProblem& p = gp.probs[tl.prob];
            const int row = tl.tm * BM + q * 32 + lane;
#pragma unroll
            for (int gq = 0; gq < 4; ++gq) {
                const int col0 = tl.tn * BN + h * 128 + gq * 32;
                if (row >= p.m || col0 >= p.n) continue;
                float* crow = p.C + (int64_t)row * p.ldc + col0;
                if (p.vec_c && col0 + 31 < p.n) {
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        float4 o = make_float4(v[gq * 32 + 4 * u], v[gq * 32 + 4 * u + 1],
                                               v[gq * 32 + 4 * u + 2], v[gq * 32 + 4 * u + 3]);
                        float4* dst = reinterpret_cast<float4*>(crow + 4 * u);
                        if (p.beta != 0.0f) {
                            const float4 old = *dst;
                            o.x = fmaf(old.x, p.beta, o.x);
                            o.y = fmaf(old.y, p.beta, o.y);
                            o.z = fmaf(old.z, p.beta, o.z);
                            o.w = fmaf(old.w, p.beta, o.w);
                        }
                        *dst = o;
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        if (col0 + j < p.n) {
                            float o = v[gq * 32 + j];
                            if (p.beta != 0.0f) o = fmaf(crow[j], p.beta, o);
                            crow[j] = o;
                        }
                    }
                }
            }
            ++it;
        }
        if (!ok) {
            abort_s = 1;
            atomicExch(gp.status, SGEMM_B200_ERR_TIMEOUT);
        }
    }

    // ------------------------------------------------------------ teardown --
    tc_fence_before();
    __syncthreads();
    if (warp == PRODUCER_WARP && lane == 0) {
        // Copies the MMA issuer never consumed (only after an abort) must land
        // before this CTA's shared memory is released.
        for (uint32_t j = consumed_s; j < issued; ++j)
            if (!mbar_wait(&full_bar[j % T::STAGES], (j / T::STAGES) & 1)) break;
    }
    if (warp == 0) {
        __syncwarp();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

// Grouped pre-pass: the A and B planes of many problems in one launch.
// Blocks [0, a_blocks) split A chunks (256 chunks of 8 k-values per block),
// blocks [a_blocks, a_blocks + b_blocks) transpose-and-split 64 x 64 tiles of
// B; a block finds its problem by binary search over the prefix sums.
struct PrepJob {
    const float* A;
    const float* B;
    uint8_t* wa;
    uint8_t* wb;
    int m, n, k, kp, lda, ldb;
    int b_tiles_n;  // 64-column tiles of B along n
    int pad;
};

struct PrepParams {
    const PrepJob* jobs;
    const int* a_prefix;  // n_jobs + 1 entries
    const int* b_prefix;
    int n_jobs;
    int a_blocks;
};

template <int PATH>
__global__ void __launch_bounds__(256) split_prepass_grouped_kernel(const PrepParams pp) {
    __shared__ float tile[64][65];
    int b = blockIdx.x;
    const bool is_a = b < pp.a_blocks;
    const int* pref = is_a ? pp.a_prefix : pp.b_prefix;
    if (!is_a) b -= pp.a_blocks;
    int lo = 0, hi = pp.n_jobs - 1;  // the last job whose first block is <= b
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pref[mid] <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    const PrepJob& j = pp.jobs[lo];
    const int local = b - pref[lo];
    if (is_a) {
        const int64_t total = (int64_t)j.m * (j.kp / 8);
        const int64_t i = (int64_t)local * 256 + threadIdx.x;
        if (i < total) split_a_chunk<PATH>(j.A, j.m, j.k, j.lda, j.kp, j.wa, i);
    } else {
        split_bt_tile<PATH>(j.B, j.k, j.n, j.ldb, j.kp, j.wb, local % j.b_tiles_n,
                            local / j.b_tiles_n, tile);
    }
}

// ------------------------------------------------- grouped split: host side --

// Host copy of a grouped launch's tables, laid out as one blob so one copy
// moves it to the device: problems | tiles | tensor maps (64-byte aligned) |
// pre-pass jobs | A prefix sums | B prefix sums.
struct GroupedTables {
    std::vector<GSProblem> probs;
    std::vector<GSTile> tiles;
    std::vector<CUtensorMap> maps;
    std::vector<PrepJob> jobs;
    std::vector<int> a_prefix, b_prefix;
    std::vector<int> k_zero;  // problems with k == 0 (plain path)
    size_t off_tiles = 0, off_maps = 0, off_jobs = 0, off_apref = 0, off_bpref = 0, bytes = 0;
};

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

template <int PATH>
static int grouped_tables(const sgemm_b200_problem* pr, void* const* ws, int count,
                          GroupedTables* out) {
    using T = Traits<PATH>;
    GroupedTables gt;
    gt.a_prefix.push_back(0);
    gt.b_prefix.push_back(0);
    for (int i = 0; i < count; ++i) {
        const sgemm_b200_problem& q = pr[i];
        if (q.m == 0 || q.n == 0) continue;
        if (q.k == 0) {
            gt.k_zero.push_back(i);
            continue;
        }
        size_t a_bytes = 0;
        workspace_bytes<PATH>(q.m, q.n, q.k, &a_bytes);
        uint8_t* wa = reinterpret_cast<uint8_t*>(
            (reinterpret_cast<uintptr_t>(ws[i]) + 1023) & ~static_cast<uintptr_t>(1023));
        uint8_t* wb = wa + a_bytes;
        const int kp = (q.k + 7) / 8 * 8;
        const int idx = (int)gt.probs.size();
        GSProblem g;
        g.m = q.m;
        g.n = q.n;
        g.k = q.k;
        g.ldc = q.ldc;
        g.alpha = q.alpha;
        g.beta = q.beta;
        g.C = q.C;
        g.vec_c = (q.ldc % 4 == 0) && (reinterpret_cast<uintptr_t>(q.C) % 16 == 0);
        g.pad = 0;
        gt.probs.push_back(g);
        CUtensorMap ma, mb;
        std::memset(&ma, 0, sizeof(ma));
        std::memset(&mb, 0, sizeof(mb));
        const CUtensorMapDataType dt =
            T::ESZ == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
        const uint64_t row = (uint64_t)kp * T::ESZ;
        if (!encode_tensor_map_3d(&ma, dt, wa, (uint64_t)q.k, (uint64_t)q.m, T::NSPLIT, row,
                                  row * (uint64_t)q.m, T::BK, BM, T::NSPLIT,
                                  CU_TENSOR_MAP_SWIZZLE_64B) ||
            !encode_tensor_map_3d(&mb, dt, wb, (uint64_t)q.k, (uint64_t)q.n, T::NSPLIT, row,
                                  row * (uint64_t)q.n, T::BK, BN, T::NSPLIT,
                                  CU_TENSOR_MAP_SWIZZLE_64B))
            return SGEMM_B200_ERR_CUDA;
        gt.maps.push_back(ma);
        gt.maps.push_back(mb);
        PrepJob j;
        j.A = q.A;
        j.B = q.B;
        j.wa = wa;
        j.wb = wb;
        j.m = q.m;
        j.n = q.n;
        j.k = q.k;
        j.kp = kp;
        j.lda = q.lda;
        j.ldb = q.ldb;
        j.b_tiles_n = div_up(q.n, 64);
        j.pad = 0;
        gt.jobs.push_back(j);
        const int64_t a_chunks = (int64_t)q.m * (kp / 8);
        gt.a_prefix.push_back(gt.a_prefix.back() + (int)((a_chunks + 255) / 256));
        gt.b_prefix.push_back(gt.b_prefix.back() + j.b_tiles_n * div_up(kp, 64));
        const int nk = div_up(q.k, T::BK);
        for (int a = 0; a < div_up(q.m, BM); ++a)
            for (int b = 0; b < div_up(q.n, BN); ++b) gt.tiles.push_back(GSTile{idx, a, b, nk});
    }
    // longest first (all tiles have the same area; their cost is their k depth)
    std::stable_sort(gt.tiles.begin(), gt.tiles.end(),
                     [](const GSTile& x, const GSTile& y) { return x.nk > y.nk; });
    gt.off_tiles = align_up(sizeof(GSProblem) * gt.probs.size(), 64);
    gt.off_maps = align_up(gt.off_tiles + sizeof(GSTile) * gt.tiles.size(), 64);
    gt.off_jobs = align_up(gt.off_maps + sizeof(CUtensorMap) * gt.maps.size(), 64);
    gt.off_apref = align_up(gt.off_jobs + sizeof(PrepJob) * gt.jobs.size(), 64);
    gt.off_bpref = align_up(gt.off_apref + sizeof(int) * gt.a_prefix.size(), 64);
    gt.bytes = align_up(gt.off_bpref + sizeof(int) * gt.b_prefix.size(), 64);
    *out = std::move(gt);
    return SGEMM_B200_OK;
}

static void pack_tables(const GroupedTables& gt, uint8_t* h) {
    std::memcpy(h, gt.probs.data(), sizeof(GSProblem) * gt.probs.size());
    std::memcpy(h + gt.off_tiles, gt.tiles.data(), sizeof(GSTile) * gt.tiles.size());
    std::memcpy(h + gt.off_maps, gt.maps.data(), sizeof(CUtensorMap) * gt.maps.size());
    std::memcpy(h + gt.off_jobs, gt.jobs.data(), sizeof(PrepJob) * gt.jobs.size());
    std::memcpy(h + gt.off_apref, gt.a_prefix.data(), sizeof(int) * gt.a_prefix.size());
    std::memcpy(h + gt.off_bpref, gt.b_prefix.data(), sizeof(int) * gt.b_prefix.size());
}

// The grouped kernel's shared-memory attribute, once per device.
template <int PATH>
static int set_grouped_attribute() {
    static std::atomic<bool> done[64];
    static std::mutex mu;
    const int dev = device_info().device;
    if (dev < 0 || dev >= 64) return SGEMM_B200_ERR_CUDA;
    if (done[dev].load(std::memory_order_acquire)) return SGEMM_B200_OK;
    std::lock_guard<std::mutex> lock(mu);
    if (!done[dev].load(std::memory_order_relaxed)) {
        const cudaError_t e =
            cudaFuncSetAttribute(split_grouped_kernel<PATH>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 Layout<PATH>::SMEM_BYTES);
        if (e != cudaSuccess) return cuda_status(e);
        done[dev].store(true, std::memory_order_release);
    }
    return SGEMM_B200_OK;
}

// Pre-pass and persistent kernel over the tables at device address d.
template <int PATH>
static int grouped_enqueue(const GroupedTables& gt, const uint8_t* d, cudaStream_t stream) {
    if (gt.tiles.empty()) return SGEMM_B200_OK;
    int st = set_grouped_attribute<PATH>();
    if (st != SGEMM_B200_OK) return st;
    PrepParams pp;
    pp.jobs = reinterpret_cast<const PrepJob*>(d + gt.off_jobs);
    pp.a_prefix = reinterpret_cast<const int*>(d + gt.off_apref);
    pp.b_prefix = reinterpret_cast<const int*>(d + gt.off_bpref);
    pp.n_jobs = (int)gt.jobs.size();
    pp.a_blocks = gt.a_prefix.back();
    const int blocks = gt.a_prefix.back() + gt.b_prefix.back();
    split_prepass_grouped_kernel<PATH><<<blocks, 256, 0, stream>>>(pp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        note_error("grouped split pre-pass launch (%d blocks): %s", blocks, cudaGetErrorString(e));
        return cuda_status(e) == SGEMM_B200_ERR_NO_MEMORY ? SGEMM_B200_ERR_NO_MEMORY
                                                           : SGEMM_B200_ERR_CUDA;
    }
    GSParams gp;
    gp.probs = reinterpret_cast<const GSProblem*>(d);
    gp.tiles = reinterpret_cast<const GSTile*>(d + gt.off_tiles);
    gp.maps = reinterpret_cast<const CUtensorMap*>(d + gt.off_maps);
    gp.status = device_status_ptr();
    gp.n_tiles = (int)gt.tiles.size();
    if (!gp.status) return SGEMM_B200_ERR_CUDA;
    const int sms = device_info().sm_count > 0 ? device_info().sm_count : 148;
    const int grid = std::min(gp.n_tiles, sms);
    split_grouped_kernel<PATH><<<grid, THREADS, Layout<PATH>::SMEM_BYTES, stream>>>(gp);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        note_error("grouped split kernel launch (%d CTAs x %d threads, %d B shared): %s", grid,
                   THREADS, Layout<PATH>::SMEM_BYTES, cudaGetErrorString(e));
        return SGEMM_B200_ERR_CUDA;
    }
    return SGEMM_B200_OK;
}

template <int PATH>
static int grouped_arena_launch(Arena* a, const sgemm_b200_problem* probs, void* const* ws,
                                int count, cudaStream_t stream) {
    GroupedTables gt;
    int st = grouped_tables<PATH>(probs, ws, count, &gt);
    if (st != SGEMM_B200_OK) return st;
    if (!gt.tiles.empty()) {
        if (gt.bytes > a->cap) {
            // grow: generous first size (64 KiB covers ~100 problems), doubling
            const size_t n = std::max({gt.bytes, a->cap * 2, (size_t)65536});
            if (a->d) cudaFreeAsync(a->d, stream);
            if (a->h) cudaFreeHost(a->h);
            a->d = nullptr;
            a->h = nullptr;
            a->cap = 0;
            cudaMemPool_t pool = library_pool();
            if (!pool) return SGEMM_B200_ERR_CUDA;
            cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&a->d), n, pool,
                                                    stream);
            if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&a->h), n);
            if (e != cudaSuccess) return cuda_status(e);
            a->cap = n;
        }
        pack_tables(gt, a->h);
        st = cuda_status(cudaMemcpyAsync(a->d, a->h, gt.bytes, cudaMemcpyHostToDevice, stream));
        if (st == SGEMM_B200_OK) st = grouped_enqueue<PATH>(gt, a->d, stream);
        if (st != SGEMM_B200_OK) return st;
    }
    for (int i : gt.k_zero) {  // C := beta * C
        const sgemm_b200_problem& q = probs[i];
        st = plain_launch(-1, q.m, q.n, 0, q.alpha, q.A, q.lda, q.B, q.ldb, q.beta, q.C, q.ldc,
                          stream);
        if (st != SGEMM_B200_OK) return st;
    }
    return SGEMM_B200_OK;
}

size_t problem_workspace_bytes(int path, int m, int n, int k) {
    if (m <= 0 || n <= 0 || k <= 0) return 0;
    return path == SGEMM_B200_PATH_BF16X6 ? workspace_bytes<SGEMM_B200_PATH_BF16X6>(m, n, k)
                                          : workspace_bytes<SGEMM_B200_PATH_TF32X3>(m, n, k);
}

int grouped_launch(Arena* a, int path, const sgemm_b200_problem* probs, void* const* ws,
                   int count, cudaStream_t stream) {
    if (!device_is_sm100()) return SGEMM_B200_ERR_UNSUPPORTED;
    if (path == SGEMM_B200_PATH_BF16X6)
        return grouped_arena_launch<SGEMM_B200_PATH_BF16X6>(a, probs, ws, count, stream);
    if (path == SGEMM_B200_PATH_TF32X3)
        return grouped_arena_launch<SGEMM_B200_PATH_TF32X3>(a, probs, ws, count, stream);
    return SGEMM_B200_ERR_INVALID_ARG;
}

void arena_release(Arena* a) {
    cudaFree(a->d);
    cudaFreeHost(a->h);
    *a = Arena();
}

}  // namespace split

int split_launch(int path, int m, int n, int k, float alpha, const float* A, int lda,
                 const float* B, int ldb, float beta, float* C, int ldc, void* ws,
                 size_t ws_bytes, cudaStream_t stream) {
    if (m == 0 || n == 0) return SGEMM_B200_OK;
    if (!device_is_sm100()) return SGEMM_B200_ERR_UNSUPPORTED;
    if (k == 0)  // C = beta*C: no products to split
        return plain_launch(-1, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream);
    const size_t need = path == SGEMM_B200_PATH_BF16X6
                            ? split::workspace_bytes<SGEMM_B200_PATH_BF16X6>(m, n, k)
                            : split::workspace_bytes<SGEMM_B200_PATH_TF32X3>(m, n, k);
    bool owned = false;
    if (!ws) {
        cudaMemPool_t pool = library_pool();
        if (!pool) return SGEMM_B200_ERR_CUDA;
        cudaError_t e = cudaMallocFromPoolAsync(&ws, need, pool, stream);
        if (e != cudaSuccess) return cuda_status(e);
        ws_bytes = need;
        owned = true;
    }
    int s;
    if (path == SGEMM_B200_PATH_BF16X6)
        s = split::launch<SGEMM_B200_PATH_BF16X6>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, ws,
                                                  ws_bytes, stream);
    else
        s = split::launch<SGEMM_B200_PATH_TF32X3>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, ws,
                                                  ws_bytes, stream);
    if (owned) cudaFreeAsync(ws, stream);
    return s;
}

}  // namespace sgb

extern "C" size_t sgemm_b200_split_workspace_size(int path, int m, int n, int k) {
    if (m <= 0 || n <= 0 || k <= 0) return 0;
    if (path == SGEMM_B200_PATH_BF16X6)
        return sgb::split::workspace_bytes<SGEMM_B200_PATH_BF16X6>(m, n, k);
    if (path == SGEMM_B200_PATH_TF32X3)
        return sgb::split::workspace_bytes<SGEMM_B200_PATH_TF32X3>(m, n, k);
    return 0;
}

extern "C" int sgemm_b200_split(int path, int m, int n, int k, const float* alpha, const float* A,
                                int lda, const float* B, int ldb, const float* beta, float* C,
                                int ldc, void* workspace, size_t workspace_bytes,
                                sgemm_b200_stream_t stream) {
    int s = sgb::check_gemm_args(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    if (s == SGEMM_B200_OK && path != SGEMM_B200_PATH_BF16X6 && path != SGEMM_B200_PATH_TF32X3)
        s = SGEMM_B200_ERR_INVALID_ARG;
    if (s == SGEMM_B200_OK)
        s = sgb::split_launch(path, m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc, workspace,
                              workspace_bytes, sgb::as_stream(stream));
    sgb::set_last_status(s);
    return s;
}

namespace sgb {
namespace split {

// One grouped launch with its workspace and tables allocated stream-ordered
// from the library pool and freed after the kernels (the table upload is a
// pageable copy, staged by the driver before the call returns).
template <int PATH>
static int grouped_oneshot(const sgemm_b200_problem* probs, int count, cudaStream_t stream) {
    cudaMemPool_t pool = library_pool();
    if (!pool) return SGEMM_B200_ERR_CUDA;
    std::vector<size_t> off(count, 0);
    size_t total = 0;
    for (int i = 0; i < count; ++i) {
        off[i] = total;
        total += align_up(problem_workspace_bytes(PATH, probs[i].m, probs[i].n, probs[i].k), 1024);
    }
    uint8_t* ws = nullptr;
    if (total) {
        const cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&ws), total, pool,
                                                      stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    std::vector<void*> wsp(count);
    for (int i = 0; i < count; ++i) wsp[i] = ws + off[i];
    GroupedTables gt;
    int st = grouped_tables<PATH>(probs, wsp.data(), count, &gt);
    uint8_t* d = nullptr;
    if (st == SGEMM_B200_OK && !gt.tiles.empty()) {
        std::vector<uint8_t> h(gt.bytes);
        pack_tables(gt, h.data());
        st = cuda_status(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&d), gt.bytes, pool,
                                                 stream));
        if (st == SGEMM_B200_OK)
            st = cuda_status(cudaMemcpyAsync(d, h.data(), gt.bytes, cudaMemcpyHostToDevice,
                                             stream));
        if (st == SGEMM_B200_OK) st = grouped_enqueue<PATH>(gt, d, stream);
    }
    for (size_t z = 0; st == SGEMM_B200_OK && z < gt.k_zero.size(); ++z) {
        const sgemm_b200_problem& q = probs[gt.k_zero[z]];
        st = plain_launch(-1, q.m, q.n, 0, q.alpha, q.A, q.lda, q.B, q.ldb, q.beta, q.C, q.ldc,
                          stream);
    }
    if (d) cudaFreeAsync(d, stream);
    if (ws) cudaFreeAsync(ws, stream);
    return st;
}

}  // namespace split
}  // namespace sgb

extern "C" int sgemm_b200_grouped_split(int path, const sgemm_b200_problem* problems, int count,
                                        sgemm_b200_stream_t stream) {
    int s = SGEMM_B200_OK;
    if (count < 0 || (count > 0 && !problems) ||
        (path != SGEMM_B200_PATH_BF16X6 && path != SGEMM_B200_PATH_TF32X3))
        s = SGEMM_B200_ERR_INVALID_ARG;
    for (int i = 0; s == SGEMM_B200_OK && i < count; ++i) {
        const sgemm_b200_problem& q = problems[i];
        s = sgb::check_gemm_args(q.m, q.n, q.k, &q.alpha, q.A, q.lda, q.B, q.ldb, &q.beta, q.C,
                                 q.ldc);
    }
    if (s == SGEMM_B200_OK && count > 0 && !sgb::device_is_sm100()) s = SGEMM_B200_ERR_UNSUPPORTED;
    if (s == SGEMM_B200_OK && count > 0)
        s = path == SGEMM_B200_PATH_BF16X6
                ? sgb::split::grouped_oneshot<SGEMM_B200_PATH_BF16X6>(problems, count,
                                                                      sgb::as_stream(stream))
                : sgb::split::grouped_oneshot<SGEMM_B200_PATH_TF32X3>(problems, count,
                                                                      sgb::as_stream(stream));
    sgb::set_last_status(s);
    return s;
}

extern "C" int sgemm_b200_grouped_split_sequential(int path, const sgemm_b200_problem* problems,
                                                   int count, sgemm_b200_stream_t stream) {
    if (count < 0 || (count > 0 && !problems)) return SGEMM_B200_ERR_INVALID_ARG;
    for (int i = 0; i < count; ++i) {
        const sgemm_b200_problem& q = problems[i];
        const int s = sgemm_b200_split(path, q.m, q.n, q.k, &q.alpha, q.A, q.lda, q.B, q.ldb,
                                       &q.beta, q.C, q.ldc, nullptr, 0, stream);
        if (s != SGEMM_B200_OK) return s;
    }
    return SGEMM_B200_OK;
}

extern "C" int sgemm_b200_gemm(int path, int m, int n, int k, const float* alpha, const float* A,
                               int lda, const float* B, int ldb, const float* beta, float* C,
                               int ldc, sgemm_b200_stream_t stream) {
    if (path == SGEMM_B200_PATH_PLAIN)
        return sgemm_b200(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream);
    return sgemm_b200_split(path, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, nullptr, 0,
                            stream);
}

// ------------------------------------------------------- allocation-free variant --
//
// sgemm_b200_split_noalloc: the split-precision GEMM for callers that may not
// allocate device memory.  Its scratch (the BF16 / TF32 operand planes the
// pre-pass writes) is a file-scope static device array of kNoAllocScratchBytes,
// so the call itself never allocates.  The array is created when this
// library's device code is loaded on a GPU and stays until the process exits.
// It holds 64 MiB of planes plus the 1 KiB a workspace reserves to align its
// base, so a problem fits exactly when sgemm_b200_split_workspace_size() is at
// most kNoAllocScratchBytes: up to m = n = k = 2048 for TF32X3 (planes of
// exactly 64 MiB) and 2361 for BF16X6.
namespace sgb {
namespace noalloc {

constexpr size_t kNoAllocPlaneBytes = size_t(64) << 20;              // 64 MiB of planes
constexpr size_t kNoAllocScratchBytes = kNoAllocPlaneBytes + 1024;  // + base alignment
static __device__ __align__(256) uint8_t g_split_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;

// Device address of the scratch array on the current device, resolved once
// per device (host code cannot use the array's name as a device address).
static void* scratch_address(int* status) {
    static void* addr[kMaxDevices] = {nullptr};
    static std::mutex mu;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        *status = SGEMM_B200_ERR_CUDA;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_split_scratch);
        if (e != cudaSuccess || !p) {
            *status = cuda_status(e == cudaSuccess ? cudaErrorInvalidSymbol : e);
            return nullptr;
        }
        addr[dev] = p;
    }
    *status = SGEMM_B200_OK;
    return addr[dev];
}

}  // namespace noalloc
}  // namespace sgb

extern "C" int sgemm_b200_split_noalloc(int path, int m, int n, int k, const float* alpha,
                                        const float* A, int lda, const float* B, int ldb,
                                        const float* beta, float* C, int ldc,
                                        sgemm_b200_stream_t stream) {
    int s = sgb::check_gemm_args(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    if (s == SGEMM_B200_OK && path != SGEMM_B200_PATH_BF16X6 && path != SGEMM_B200_PATH_TF32X3)
        s = SGEMM_B200_ERR_INVALID_ARG;
    if (s == SGEMM_B200_OK && m > 0 && n > 0 && k > 0 &&
        sgemm_b200_split_workspace_size(path, m, n, k) > sgb::noalloc::kNoAllocScratchBytes)
        s = SGEMM_B200_ERR_NO_MEMORY;  // the fixed scratch cannot hold this problem's planes
    void* scratch = nullptr;
    if (s == SGEMM_B200_OK) scratch = sgb::noalloc::scratch_address(&s);
    if (s == SGEMM_B200_OK)
        s = sgb::split_launch(path, m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc, scratch,
                              sgb::noalloc::kNoAllocScratchBytes, sgb::as_stream(stream));
    sgb::set_last_status(s);
    return s;
}
