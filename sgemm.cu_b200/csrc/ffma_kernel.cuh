// ffma_kernel.cuh — the plain FP32 path: register-blocked FFMA SGEMM for sm_100a.
//
// Replaces the reference's sgemm_128x128x8 / sgemm_128x256x8
// (src/kernels/128x128x8.cuh, src/kernels/128x256x8.cuh).  Same contract and
// same arithmetic per C element:
//     acc = 0; for p = 0..k-1 in increasing order: acc = fma(A[i,p], B[p,j], acc)
//     acc = acc * alpha;  C[i,j] = beta != 0 ? fma(C[i,j], beta, acc) : acc
// (reference: 128x256x8.cuh:224-239 for the chain, :331-337 for alpha,
// :365-380 for the beta branch), so outputs are bit-identical.  Zero-filled
// k padding adds exact +0 terms, as the reference's padded first block does
// (128x256x8.cuh:87-116).
//
// B200 design (not the reference's):
//  - CTA tile BM x BN with a 32-deep k block, STAGES-deep ring of stages in
//    shared memory filled by TMA (one elected thread, mbarrier completion) or,
//    for strides that TMA cannot describe (lda/ldb not a multiple of 4),
//    by 4-byte cp.async with zero fill;
//  - A is kept k-contiguous ([m][32] rows of 128 B) with the 128-byte XOR
//    swizzle TMA applies, so a thread reads 4 k-values of one row with one
//    conflict-free 128-bit shared load (instead of transposing A in smem);
//  - B is kept [32][BN]; each 128-bit load is broadcast to the 4 lanes that
//    share a column group (warp-level operand broadcast);
//  - thread tile TM (m, 8 or 7) x TN (n); lanes 4 (m) x 8 (n); warps WM x WN;
//  - the FMAs are packed (fma.rn.f32x2, two columns of a row per
//    instruction): the FP32 pipe, not instruction issue, becomes the limit;
//  - epilogue straight from registers with float4 stores: for a fixed
//    register group a warp writes 4 rows x 128 contiguous bytes.
#pragma once

#include <cstdint>

#include "ptx.cuh"

namespace sgb {
namespace ffma {

enum Loader { kLoaderTma = 0, kLoaderAsync4 = 1 };

template <int BM_, int BN_, int WM_, int WN_, int TN_, int STAGES_, int LOADER_, int MINB_ = 1,
          int K4U_ = 8, int PRODUCER_ = 0, int TM_ = 8>
struct Cfg {
    static constexpr int BM = BM_, BN = BN_, WM = WM_, WN = WN_, TN = TN_, STAGES = STAGES_;
    static constexpr int LOADER = LOADER_;
    static constexpr int MINB = MINB_;  // resident CTAs per SM the register budget targets
    static constexpr int K4U = K4U_;    // unroll of the 8 four-deep k steps of a k block
    // PRODUCER: one extra warp issues the TMA loads, and the compute warps free
    // each stage through a per-stage "empty" mbarrier instead of a CTA barrier.
    static constexpr int PRODUCER = PRODUCER_;
    static constexpr int BK = 32;  // one 128-byte row of A per k block
    // rows per thread: 8, or 7 for the tile whose 28 rows split a 1024-row
    // problem into one CTA per SM
    static constexpr int TM = TM_;
    static constexpr int WROWS = 4 * TM;  // rows of a warp's tile (4 lanes x TM)
    static constexpr int COMPUTE_THREADS = 32 * WM * WN;
    static constexpr int THREADS = COMPUTE_THREADS + (PRODUCER ? 32 : 0);
    static_assert(!PRODUCER || LOADER_ == 0, "the producer warp issues TMA loads");
    static_assert(BM == WM * WROWS, "4 lanes x TM rows per warp along m");
    static_assert(BN == WN * 8 * TN, "8 lanes x TN columns per warp along n");
    static_assert(TN % 4 == 0, "columns come in float4 groups");
    static constexpr int A_TX = BM * BK * 4;  // bytes one A box brings
    // A's region in a stage, rounded up to the 1024-byte swizzle atom so that
    // B (and the next stage) start on one
    static constexpr int A_BYTES = (A_TX + 1023) / 1024 * 1024;
    static constexpr int B_BYTES = BK * BN * 4;
    static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;  // stride between stages
    static constexpr int STAGE_TX = A_TX + B_BYTES;        // bytes a stage's copies bring
    static_assert(A_BYTES % 1024 == 0 && STAGE_BYTES % 1024 == 0, "1024-byte swizzle atoms");
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;  // + alignment slack
};


// Lane -> (lm, ln) on the 4 (m) x 8 (n) lane grid: lm = lane % 4,
// ln = lane / 4, so a quarter-warp owns 4 rows x 2 column groups.  The map
// only decides which thread owns which outputs (every output keeps its own
// k-ordered FMA chain).  Measured on a B200 at 4096..16384 against
// lm = lane / 8 (a quarter-warp on one row) and a 2 x 4 quarter-warp block:
// this one is 0.5-2.6% faster although the 2 x 4 block needs fewer shared
// wavefronts (2 instead of 3 per 128-bit load) -- shared bandwidth is not
// what limits this kernel.
__device__ __forceinline__ void lane_coords(int lane, int& lm, int& ln) {
    lm = lane & 3;
    ln = lane >> 2;
}

// Grouped rasterisation: 8 tile-rows share a band so concurrently resident
// CTAs reuse A rows and B columns out of L2.
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

// A's shared-memory coordinates for a thread: its first row of the tile is
// r0 = wm * WROWS + lm and its i-th row r0 + 4i, at byte r0 * 128 + i * 512.
// The 128-byte swizzle XORs a row's 16-byte chunk index with row % 8, which
// along i alternates between xa0 (even i) and xa1 (odd i).
template <class C>
__device__ __forceinline__ void a_coords(int wm, int lm, uint32_t& a_base, uint32_t& xa0,
                                         uint32_t& xa1) {
    const int r0 = wm * C::WROWS + lm;
    a_base = static_cast<uint32_t>(r0 * 128);
    xa0 = static_cast<uint32_t>(r0 & 7) << 4;
    xa1 = static_cast<uint32_t>((r0 + 4) & 7) << 4;
}

// Fragment loads of one k block: A rows for the 4-deep step k4 (4 k-values of
// each of the thread's 8 rows) and B columns for one k.
template <class C>
__device__ __forceinline__ void load_a_frag(const uint8_t* __restrict__ As, uint32_t a_base,
                                            uint32_t xa0, uint32_t xa1, int k4,
                                            float4 (&a)[C::TM]) {
#pragma unroll
    for (int i = 0; i < C::TM; ++i) {
        const uint32_t x = (i & 1) ? xa1 : xa0;
        const uint32_t off = a_base + i * 4 * 128 + ((static_cast<uint32_t>(k4) << 4) ^ x);
        a[i] = *reinterpret_cast<const float4*>(As + off);
    }
}

template <class C>
__device__ __forceinline__ void load_b_frag(const uint8_t* __restrict__ Bs, uint32_t b_base, int k,
                                            float4 (&b)[C::TN / 4]) {
#pragma unroll
    for (int g = 0; g < C::TN / 4; ++g)
        b[g] = *reinterpret_cast<const float4*>(Bs + k * C::BN * 4 + b_base + g * 128);
}

// Accumulate one 32-deep k block held in shared memory: A fragments for a
// 4-deep step at its start, B per k (the compiler schedules the loads).  Each
// element accumulates over k in increasing order with one FMA per term.
template <class C>
__device__ __forceinline__ void compute_stage(const uint8_t* __restrict__ As,
                                                     const uint8_t* __restrict__ Bs,
                                                     uint32_t a_base, uint32_t xa0, uint32_t xa1,
                                                     uint32_t b_base, float (&acc)[C::TM][C::TN]) {
#pragma unroll C::K4U
    for (int k4 = 0; k4 < C::BK / 4; ++k4) {
        float4 a[C::TM];
#pragma unroll
        for (int i = 0; i < C::TM; ++i) {
            const uint32_t x = (i & 1) ? xa1 : xa0;
            const uint32_t off = a_base + i * 4 * 128 + ((static_cast<uint32_t>(k4) << 4) ^ x);
            a[i] = *reinterpret_cast<const float4*>(As + off);
        }
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            float4 b[C::TN / 4];
#pragma unroll
            for (int g = 0; g < C::TN / 4; ++g)
                b[g] = *reinterpret_cast<const float4*>(Bs + (k4 * 4 + kk) * C::BN * 4 + b_base +
                                                        g * 128);
            // Outer product with packed FP32 FMAs (fma.rn.f32x2): each
            // instruction updates two neighbouring columns of one row,
            // {c[i][j], c[i][j+1]} += {a_i, a_i} * {b_j, b_j+1}, with one
            // round-to-nearest FMA per element -- the same arithmetic as two
            // fmaf calls, in half the issue slots.  Rows run in serpentine
            // order (row i left to right, row i+1 right to left) so
            // consecutive instructions share an operand at every turn.
            // Measured on a B200: +7.5% at 8192^3 over one fmaf per element
            // (which was issue-bound); serpentine order +0.7% over row-major.
            float av[C::TM], bv[C::TN];
#pragma unroll
            for (int i = 0; i < C::TM; ++i)
                av[i] = kk == 0 ? a[i].x : kk == 1 ? a[i].y : kk == 2 ? a[i].z : a[i].w;
#pragma unroll
            for (int g = 0; g < C::TN / 4; ++g) {
                bv[4 * g + 0] = b[g].x;
                bv[4 * g + 1] = b[g].y;
                bv[4 * g + 2] = b[g].z;
                bv[4 * g + 3] = b[g].w;
            }
#pragma unroll
            for (int i = 0; i < C::TM; ++i) {
                const float2 a2 = make_float2(av[i], av[i]);
#pragma unroll
                for (int pp = 0; pp < C::TN / 2; ++pp) {
                    const int q = (i & 1) ? C::TN / 2 - 1 - pp : pp;
                    float2 c = make_float2(acc[i][2 * q], acc[i][2 * q + 1]);
                    c = __ffma2_rn(a2, make_float2(bv[2 * q], bv[2 * q + 1]), c);
                    acc[i][2 * q] = c.x;
                    acc[i][2 * q + 1] = c.y;
                }
            }
        }
    }
}

// Operand and output views of one GEMM, shared by the single-problem kernel
// and the grouped persistent kernel.
struct Operands {
    int m, n, k;
    int lda, ldb, ldc;
    float alpha, beta;
    const float* A;
    const float* B;
    float* C;
    int vec_c;
};

// cp.async loader for one k block (any stride, any alignment).
template <class C>
__device__ __forceinline__ void load_stage_async4(const Operands& p, uint8_t* As, uint8_t* Bs,
                                                  int m0, int n0, int k0, int tid) {
    const uint32_t as = smem_u32(As), bs = smem_u32(Bs);
    constexpr int A_ELEMS = C::BM * C::BK;
#pragma unroll 4
    for (int e = tid; e < A_ELEMS; e += C::THREADS) {
        const int r = e >> 5, c = e & 31;
        const bool ok = (m0 + r < p.m) && (k0 + c < p.k);
        const float* src = ok ? p.A + (int64_t)(m0 + r) * p.lda + (k0 + c) : p.A;
        const uint32_t dst = as + r * 128 + ((((c >> 2) ^ (r & 7)) << 4) | ((c & 3) << 2));
        cp_async_4_zfill(dst, src, ok);
    }
    constexpr int B_ELEMS = C::BK * C::BN;
#pragma unroll 4
    for (int e = tid; e < B_ELEMS; e += C::THREADS) {
        const int r = e / C::BN, c = e % C::BN;
        const bool ok = (k0 + r < p.k) && (n0 + c < p.n);
        const float* src = ok ? p.B + (int64_t)(k0 + r) * p.ldb + (n0 + c) : p.B;
        cp_async_4_zfill(bs + (r * C::BN + c) * 4, src, ok);
    }
}

// Thread (wm, wn, lm, ln) owns rows m0 + WROWS wm + lm + 4i (i < TM) and the
// float4 column groups n0 + wn*8*TN + 4ln + 32g (g < TN/4).  One row at a
// time, each C load right before its store.
template <class C>
__device__ __forceinline__ void epilogue_rows(const Operands& p, int m0, int n0, int wm, int wn,
                                              int lm, int ln, const float (&acc)[C::TM][C::TN]) {
    const int col0 = n0 + wn * 8 * C::TN + ln * 4;
#pragma unroll
    for (int i = 0; i < C::TM; ++i) {
        const int row = m0 + wm * C::WROWS + lm + 4 * i;
        if (row >= p.m) continue;
        float* crow = p.C + (int64_t)row * p.ldc;
#pragma unroll
        for (int g = 0; g < C::TN / 4; ++g) {
            const int col = col0 + 32 * g;
            float v[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) v[e] = __fmul_rn(acc[i][4 * g + e], p.alpha);
            if (p.vec_c && col + 3 < p.n) {
                float4* dst = reinterpret_cast<float4*>(crow + col);
                if (p.beta != 0.0f) {
                    const float4 o = *dst;
                    v[0] = fmaf(o.x, p.beta, v[0]);
                    v[1] = fmaf(o.y, p.beta, v[1]);
                    v[2] = fmaf(o.z, p.beta, v[2]);
                    v[3] = fmaf(o.w, p.beta, v[3]);
                }
                *dst = make_float4(v[0], v[1], v[2], v[3]);
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    if (col + e < p.n) {
                        float out = v[e];
                        if (p.beta != 0.0f) out = fmaf(crow[col + e], p.beta, out);
                        crow[col + e] = out;
                    }
                }
            }
        }
    }
}

// The same outputs with the C loads batched: with beta != 0 every C value a
// chunk of rows needs is loaded before the chunk's first store.  A store to C
// may alias a later load of C as far as the compiler knows, so in
// epilogue_rows each load waits for the store before it -- one DRAM round
// trip per row, which on a lone CTA per SM is ~12% of a 1024^3 GEMM; a chunk
// of BATCH values pays one.  The arithmetic per element is unchanged:
// acc * alpha, then fma(C, beta, .).  Measured on a B200 against
// epilogue_rows, same bits: beta = 0.5 +14% at 1000^3 and 1024^3, +2.6% at
// 2048^3 and 3001^3, +0.6% at 4096^3 and 5003^3, level at 8192^3; beta = 0
// unchanged.  epilogue() takes BATCH 0 for epilogue_rows: the grouped
// kernel keeps it, since the batch's registers push that kernel (168 at
// three CTAs per SM) into spills and made the 512-problem mix 2% slower.
template <class C, int BATCH>
__device__ __forceinline__ void epilogue_batched(const Operands& op, int m0, int n0, int wm,
                                                 int wn, int lm, int ln,
                                                 const float (&acc)[C::TM][C::TN]) {
    // a private copy: the problem description may sit in global memory, where
    // each store to C would otherwise force it to be read again
    const Operands p = op;
    const int col0 = n0 + wn * 8 * C::TN + ln * 4;
    // rows per chunk: the chunk's BATCH old C values live in registers
    constexpr int RC = BATCH / C::TN > 0 ? BATCH / C::TN : 1;
#pragma unroll
    for (int i0 = 0; i0 < C::TM; i0 += RC) {
        float4 old[RC][C::TN / 4];
        if (p.beta != 0.0f) {
#pragma unroll
            for (int ii = 0; ii < RC; ++ii) {
                const int i = i0 + ii;
                if (i >= C::TM) break;
                const int row = m0 + wm * C::WROWS + lm + 4 * i;
#pragma unroll
                for (int g = 0; g < C::TN / 4; ++g) {
                    const int col = col0 + 32 * g;
                    old[ii][g] = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (row < p.m && p.vec_c && col + 3 < p.n)
                        old[ii][g] = *reinterpret_cast<const float4*>(p.C + (int64_t)row * p.ldc +
                                                                      col);
                }
            }
        }
#pragma unroll
        for (int ii = 0; ii < RC; ++ii) {
            const int i = i0 + ii;
            if (i >= C::TM) break;
            const int row = m0 + wm * C::WROWS + lm + 4 * i;
            if (row >= p.m) continue;
            float* crow = p.C + (int64_t)row * p.ldc;
#pragma unroll
            for (int g = 0; g < C::TN / 4; ++g) {
                const int col = col0 + 32 * g;
                float v[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) v[e] = __fmul_rn(acc[i][4 * g + e], p.alpha);
                if (p.vec_c && col + 3 < p.n) {
                    if (p.beta != 0.0f) {
                        const float4 o = old[ii][g];
                        v[0] = fmaf(o.x, p.beta, v[0]);
                        v[1] = fmaf(o.y, p.beta, v[1]);
                        v[2] = fmaf(o.z, p.beta, v[2]);
                        v[3] = fmaf(o.w, p.beta, v[3]);
                    }
                    *reinterpret_cast<float4*>(crow + col) = make_float4(v[0], v[1], v[2], v[3]);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        if (col + e < p.n) {
                            float out = v[e];
                            if (p.beta != 0.0f) out = fmaf(crow[col + e], p.beta, out);
                            crow[col + e] = out;
                        }
                    }
                }
            }
        }
    }
}

template <class C, int BATCH = 32>
__device__ __forceinline__ void epilogue(const Operands& p, int m0, int n0, int wm, int wn,
                                         int lm, int ln, const float (&acc)[C::TM][C::TN]) {
    if constexpr (BATCH == 0)
        epilogue_rows<C>(p, m0, n0, wm, wn, lm, ln, acc);
    else
        epilogue_batched<C, BATCH>(p, m0, n0, wm, wn, lm, ln, acc);
}

// Epilogue for C rows that are not 16-byte aligned (ldc % 4 != 0 or an
// unaligned base), where float4 accesses are impossible and per-thread
// scalar accesses would touch 4 rows x 4 sectors per warp instruction for
// 128 useful bytes.  Each warp first parks its WROWS x (8 TN) outputs in shared
// memory (the stage ring, free once the main loop is done), then walks its
// rows with consecutive lanes on consecutive columns: one 128-byte row
// segment per instruction.  The arithmetic per element is the epilogue's
// (acc * alpha, then fma(C, beta, .)); only the thread that does it changes.
// The caller must have made every warp finish reading the ring.
template <class C, int BATCH = 32>
__device__ __forceinline__ void epilogue_staged(const Operands& p, int m0, int n0, int wm, int wn,
                                                int lm, int ln, int warp, int lane,
                                                const float (&acc)[C::TM][C::TN], uint8_t* smem) {
    constexpr int W = 8 * C::TN;  // columns of a warp's tile
    constexpr int LD = W + 8;     // row pitch: 8 banks between rows, conflict-free float4 stores
    static_assert((C::COMPUTE_THREADS / 32) * C::WROWS * LD * 4 <= C::STAGES * C::STAGE_BYTES,
                  "the staged tile fits in the stage ring");
    float* buf = reinterpret_cast<float*>(smem) + warp * C::WROWS * LD;
#pragma unroll
    for (int i = 0; i < C::TM; ++i)
#pragma unroll
        for (int g = 0; g < C::TN / 4; ++g)
            *reinterpret_cast<float4*>(buf + (lm + 4 * i) * LD + 4 * ln + 32 * g) =
                make_float4(acc[i][4 * g], acc[i][4 * g + 1], acc[i][4 * g + 2], acc[i][4 * g + 3]);
    __syncwarp();
    const int col0 = n0 + wn * W;
    if constexpr (BATCH == 0) {  // one row at a time
        for (int r = 0; r < C::WROWS; ++r) {
            const int row = m0 + wm * C::WROWS + r;
            if (row >= p.m) break;
            float* crow = p.C + (int64_t)row * p.ldc;
#pragma unroll
            for (int t = 0; t < W / 32; ++t) {
                const int col = col0 + lane + 32 * t;
                if (col < p.n) {
                    float v = __fmul_rn(buf[r * LD + lane + 32 * t], p.alpha);
                    if (p.beta != 0.0f) v = fmaf(crow[col], p.beta, v);
                    crow[col] = v;
                }
            }
        }
        return;
    }
    // rows in chunks of 8 whose C values are all loaded before the chunk's
    // first store (see epilogue: one DRAM round trip per chunk, not per row)
    constexpr int RC = 8;
    for (int r0 = 0; r0 < C::WROWS; r0 += RC) {
        float old[RC][W / 32];
        if (p.beta != 0.0f) {
#pragma unroll
            for (int rr = 0; rr < RC; ++rr) {
                const int row = m0 + wm * C::WROWS + r0 + rr;
#pragma unroll
                for (int t = 0; t < W / 32; ++t) {
                    const int col = col0 + lane + 32 * t;
                    old[rr][t] = (r0 + rr < C::WROWS && row < p.m && col < p.n)
                                     ? p.C[(int64_t)row * p.ldc + col]
                                     : 0.0f;
                }
            }
        }
#pragma unroll
        for (int rr = 0; rr < RC; ++rr) {
            const int r = r0 + rr;
            const int row = m0 + wm * C::WROWS + r;
            if (r >= C::WROWS || row >= p.m) break;
            float* crow = p.C + (int64_t)row * p.ldc;
#pragma unroll
            for (int t = 0; t < W / 32; ++t) {
                const int col = col0 + lane + 32 * t;
                if (col < p.n) {
                    float v = __fmul_rn(buf[r * LD + lane + 32 * t], p.alpha);
                    if (p.beta != 0.0f) v = fmaf(old[rr][t], p.beta, v);
                    crow[col] = v;
                }
            }
        }
    }
}

// Barrier over the compute warps only (the producer warp, if any, has left).
template <class C>
__device__ __forceinline__ void compute_barrier() {
    if constexpr (C::PRODUCER)
        asm volatile("bar.sync 1, %0;" ::"n"(C::COMPUTE_THREADS) : "memory");
    else
        __syncthreads();
}

// The epilogue for any C: float4 stores straight from registers when C rows
// are 16-byte aligned, else the shared-memory staged form.  Called by every
// compute thread of the CTA (the staged form has a barrier).
template <class C, int BATCH = 32>
__device__ __forceinline__ void epilogue_any(const Operands& p, int m0, int n0, int wm, int wn,
                                             int lm, int ln, const float (&acc)[C::TM][C::TN],
                                             uint8_t* smem) {
    if (p.vec_c) {
        epilogue<C, BATCH>(p, m0, n0, wm, wn, lm, ln, acc);
    } else {
        compute_barrier<C>();  // every warp is done reading the stage ring
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        epilogue_staged<C, BATCH>(p, m0, n0, wm, wn, lm, ln, warp, lane, acc, smem);
    }
}

struct Params {
    Operands op;  // vec_c: C rows are 16-byte aligned (ldc % 4 == 0 and C aligned)
    int* status;
    int tiles_m, tiles_n;
    // Accumulators carried between launches over consecutive k ranges (host
    // pipeline): acc_in, when set, holds the unscaled sums of the k range
    // before this one (row-major m x n, pitch ld_acc) and seeds every
    // accumulator; acc_out, when set, receives this launch's unscaled sums
    // instead of the alpha/beta epilogue (C is neither read nor written).
    // Both 16-byte aligned with ld_acc % 4 == 0.
    const float* acc_in;
    float* acc_out;
    int ld_acc;
};

// Thread (wm, wn, lm, ln) moves its accumulators between registers and an
// m x n row-major buffer: acc[i][4g+e] is element (m0 + WROWS wm + lm + 4i,
// n0 + 8 TN wn + 4 ln + 32 g + e).  A sum resumed from the buffer continues
// the same k-ordered FMA chain, so a product computed over k ranges that
// start on whole 32-deep k blocks has the bits of the product in one launch.
template <class C, bool STORE>
__device__ __forceinline__ void acc_move(const Operands& p, const float* in, float* out, int ld,
                                         int m0, int n0, int wm, int wn, int lm, int ln,
                                         float (&acc)[C::TM][C::TN]) {
    const int col0 = n0 + wn * 8 * C::TN + ln * 4;
#pragma unroll
    for (int i = 0; i < C::TM; ++i) {
        const int row = m0 + wm * C::WROWS + lm + 4 * i;
        if (row >= p.m) continue;
#pragma unroll
        for (int g = 0; g < C::TN / 4; ++g) {
            const int col = col0 + 32 * g;
            const int64_t off = (int64_t)row * ld + col;
            if (col + 3 < p.n) {
                if constexpr (STORE) {
                    *reinterpret_cast<float4*>(out + off) =
                        make_float4(acc[i][4 * g], acc[i][4 * g + 1], acc[i][4 * g + 2],
                                    acc[i][4 * g + 3]);
                } else {
                    const float4 v = *reinterpret_cast<const float4*>(in + off);
                    acc[i][4 * g] = v.x;
                    acc[i][4 * g + 1] = v.y;
                    acc[i][4 * g + 2] = v.z;
                    acc[i][4 * g + 3] = v.w;
                }
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    if (col + e < p.n) {
                        if constexpr (STORE)
                            out[off + e] = acc[i][4 * g + e];
                        else
                            acc[i][4 * g + e] = in[off + e];
                    }
                }
            }
        }
    }
}

// The end of a tile: the unscaled sums to acc_out, or the epilogue to C.
template <class C>
__device__ __forceinline__ void finish_tile(const Params& p, int m0, int n0, int wm, int wn,
                                            int lm, int ln, float (&acc)[C::TM][C::TN],
                                            uint8_t* smem) {
    if (p.acc_out)
        acc_move<C, true>(p.op, nullptr, p.acc_out, p.ld_acc, m0, n0, wm, wn, lm, ln, acc);
    else
        epilogue_any<C>(p.op, m0, n0, wm, wn, lm, ln, acc, smem);
}

template <class C>
__global__ void __launch_bounds__(C::THREADS, C::MINB)
    ffma_gemm_kernel(const __grid_constant__ CUtensorMap tmA,
                     const __grid_constant__ CUtensorMap tmB, const Params p) {
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[C::STAGES];
    __shared__ __align__(8) uint64_t empty_bar[C::PRODUCER ? C::STAGES : 1];
    uint8_t* smem = align_smem_1024(smem_raw);

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;

    if constexpr (C::PRODUCER) {
        int tm, tn;
        tile_coords(blockIdx.x, p.tiles_m, p.tiles_n, tm, tn);
        const int nk = (p.op.k + C::BK - 1) / C::BK;
        if (tid == 0) {
            for (int s = 0; s < C::STAGES; ++s) {
                mbar_init(&full_bar[s], 1);
                mbar_init(&empty_bar[s], C::WM * C::WN);  // one arrival per compute warp
            }
            fence_barrier_init();
        }
        __syncthreads();  // the only CTA-wide barrier: barriers initialised
        if (warp == C::WM * C::WN) {
            // ------------------------------------------------ TMA producer --
            if (lane == 0 && nk > 0) {
                tma_prefetch_desc(&tmA);
                tma_prefetch_desc(&tmB);
                int kb = 0;
                for (; kb < nk; ++kb) {
                    const int s = kb % C::STAGES;
                    if (kb >= C::STAGES &&
                        !mbar_wait(&empty_bar[s], ((kb / C::STAGES) - 1) & 1)) {
                        atomicExch(p.status, SGEMM_B200_ERR_TIMEOUT);
                        break;
                    }
                    // The compute warps' generic-proxy reads of the stage,
                    // acquired through the empty barrier, before the
                    // async-proxy (TMA) writes that refill it.  Without this
                    // fence a warp of the 28 x 256 tile occasionally took one
                    // k block's products from the refill (one warp's 28 x 32
                    // patch of C wrong, under concurrent launches on a B200).
                    if (kb >= C::STAGES) fence_proxy_async_shared();
                    uint8_t* st = smem + s * C::STAGE_BYTES;
                    mbar_arrive_expect_tx(&full_bar[s], C::STAGE_TX);
                    tma_load_2d(st, &tmA, &full_bar[s], kb * C::BK, tm * C::BM);
                    tma_load_2d(st + C::A_BYTES, &tmB, &full_bar[s], tn * C::BN, kb * C::BK);
                }
                // Copies still in flight land before the CTA's smem is released
                // (the compute warps may have given up on a stage).
                for (int j = (kb > C::STAGES ? kb - C::STAGES : 0); j < kb; ++j)
                    if (!mbar_wait(&full_bar[j % C::STAGES], (j / C::STAGES) & 1)) break;
            }
            return;
        }
        const int wm = warp / C::WN, wn = warp % C::WN;
        int lm, ln;
        lane_coords(lane, lm, ln);
        const int m0 = tm * C::BM, n0 = tn * C::BN;
        uint32_t a_base, xa0, xa1;
        a_coords<C>(wm, lm, a_base, xa0, xa1);
        const uint32_t b_base = static_cast<uint32_t>((wn * 8 * C::TN + ln * 4) * 4);
        float acc[C::TM][C::TN];
#pragma unroll
        for (int i = 0; i < C::TM; ++i)
#pragma unroll
            for (int j = 0; j < C::TN; ++j) acc[i][j] = 0.0f;
        if (p.acc_in)
            acc_move<C, false>(p.op, p.acc_in, nullptr, p.ld_acc, m0, n0, wm, wn, lm, ln, acc);
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % C::STAGES;
            if (!mbar_wait(&full_bar[s], (kb / C::STAGES) & 1)) {
                if (lane == 0) atomicExch(p.status, SGEMM_B200_ERR_TIMEOUT);
                return;
            }
            const uint8_t* st = smem + s * C::STAGE_BYTES;
            compute_stage<C>(st, st + C::A_BYTES, a_base, xa0, xa1, b_base, acc);
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty_bar[s]);  // this warp is done with the stage
        }
        finish_tile<C>(p, m0, n0, wm, wn, lm, ln, acc, smem);
        return;
    }

    const int wm = warp / C::WN, wn = warp % C::WN;
    int lm, ln;
    lane_coords(lane, lm, ln);

    int tm, tn;
    tile_coords(blockIdx.x, p.tiles_m, p.tiles_n, tm, tn);
    const int m0 = tm * C::BM, n0 = tn * C::BN;
    const int nk = (p.op.k + C::BK - 1) / C::BK;

    // Per-thread shared-memory offsets (bytes within a stage).
    uint32_t a_base, xa0, xa1;
    a_coords<C>(wm, lm, a_base, xa0, xa1);
    const uint32_t b_base = static_cast<uint32_t>((wn * 8 * C::TN + ln * 4) * 4);

    float acc[C::TM][C::TN];
#pragma unroll
    for (int i = 0; i < C::TM; ++i)
#pragma unroll
        for (int j = 0; j < C::TN; ++j) acc[i][j] = 0.0f;
    if (p.acc_in)
        acc_move<C, false>(p.op, p.acc_in, nullptr, p.ld_acc, m0, n0, wm, wn, lm, ln, acc);

    if constexpr (C::LOADER == kLoaderTma) {
        int issued = 0;
        auto issue = [&](int kb) {
            const int s = kb % C::STAGES;
            uint8_t* st = smem + s * C::STAGE_BYTES;
            mbar_arrive_expect_tx(&full_bar[s], C::STAGE_TX);
            tma_load_2d(st, &tmA, &full_bar[s], kb * C::BK, m0);
            tma_load_2d(st + C::A_BYTES, &tmB, &full_bar[s], n0, kb * C::BK);
        };
        if (tid == 0) {
            for (int s = 0; s < C::STAGES; ++s) mbar_init(&full_bar[s], 1);
            fence_barrier_init();
            if (nk > 0) {
                tma_prefetch_desc(&tmA);
                tma_prefetch_desc(&tmB);
            }
        }
        __syncthreads();
        if (tid == 0) {
            for (; issued < C::STAGES && issued < nk; ++issued) issue(issued);
        }
        int kb = 0;
        bool failed = false;
        for (; kb < nk; ++kb) {
            const int s = kb % C::STAGES;
            const bool ok = mbar_wait(&full_bar[s], (kb / C::STAGES) & 1);
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            // Every thread finished block kb-1, so its stage ((kb-1) % STAGES,
            // which is where block kb-1+STAGES == issued lands) may be refilled.
            if (tid == 0 && kb > 0 && issued < nk) {
                // every thread's generic-proxy reads of the stage (ordered by the
                // barrier) before the async-proxy (TMA) writes that refill it
                fence_proxy_async_shared();
                issue(issued++);
            }
            const uint8_t* st = smem + s * C::STAGE_BYTES;
            compute_stage<C>(st, st + C::A_BYTES, a_base, xa0, xa1, b_base, acc);
        }
        if (failed) {
            if (tid == 0) {
                atomicExch(p.status, SGEMM_B200_ERR_TIMEOUT);
                // Let copies still in flight land before the CTA's smem is released.
                for (int j = kb; j < issued; ++j)
                    if (!mbar_wait(&full_bar[j % C::STAGES], (j / C::STAGES) & 1)) break;
            }
            return;
        }
    } else {
#pragma unroll
        for (int s = 0; s < C::STAGES - 1; ++s) {
            if (s < nk) {
                uint8_t* st = smem + s * C::STAGE_BYTES;
                load_stage_async4<C>(p.op, st, st + C::A_BYTES, m0, n0, s * C::BK, tid);
            }
            cp_async_commit();
        }
        for (int kb = 0; kb < nk; ++kb) {
            cp_async_wait<C::STAGES - 2>();
            __syncthreads();
            const int nxt = kb + C::STAGES - 1;
            if (nxt < nk) {
                uint8_t* st = smem + (nxt % C::STAGES) * C::STAGE_BYTES;
                load_stage_async4<C>(p.op, st, st + C::A_BYTES, m0, n0, nxt * C::BK, tid);
            }
            cp_async_commit();
            const uint8_t* st = smem + (kb % C::STAGES) * C::STAGE_BYTES;
            compute_stage<C>(st, st + C::A_BYTES, a_base, xa0, xa1, b_base, acc);
        }
        cp_async_wait<0>();
    }

    finish_tile<C>(p, m0, n0, wm, wn, lm, ln, acc, smem);
}

}  // namespace ffma
}  // namespace sgb
