// grouped.cu — persistent grouped FP32 GEMM: many independent (M, N, K)
// problems in one launch, plus its autotuner.
//
// No reference counterpart (the reference launches one GEMM per call,
// src/sgemm.cuh:19-48); every problem keeps sgemm()'s contract.
//
// Design:
//  - The plan flattens every problem into work items (tile_m, tile_n, k
//    split), sorted longest-first so the tail of the launch is short items.
//  - Persistent 4-warp CTAs (2 or 3 per SM) claim items with an atomic
//    counter and run the same FFMA core as the plain path on each: one of two
//    tile shapes (128x64 or 64x128, 8 x 8 thread tiles) and one of two
//    loaders (TMA with per-problem tensor maps kept in global memory, or
//    4-byte cp.async for strides TMA cannot describe), chosen per problem at
//    plan time.
//  - Items with split == 1 run the plain path's exact arithmetic, so their
//    results equal sgemm_b200's bit for bit.  Split-K items write partial sums
//    to a workspace; the last split of a tile to finish (atomic ticket) adds
//    the partials in split order 0, 1, 2, ... and applies alpha/beta, so the
//    result is deterministic and independent of scheduling.
//  - The launch (counter reset + kernel) is captured once into a CUDA graph
//    and replayed.
//  - Tile shape, split-K and stage count per size bucket come from the
//    autotuner (sgemm_b200_autotune_grouped), persisted as JSON keyed by the
//    device name and SM count.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "common.h"
#include "ffma_kernel.cuh"
#include "grouped.h"
#include "plain.h"

namespace sgb {
namespace grouped {

using ffma::Operands;

// Three tile shapes of the plain path's 4-warp FFMA core share one kernel
// (same thread count, one 24 KB shared-memory slot per stage): 128 x 64 and
// 64 x 128 with 8 x 8 threads, and 32 x 128 with 8 x 4 threads for problems
// only a few rows tall, whose rows a 64- or 128-row tile would mostly pad
// with zeros.  3 stages fit 3 CTAs per SM, 4 stages fit 2.
template <int S>
using CfgT = ffma::Cfg<128, 64, 4, 1, 8, S, ffma::kLoaderTma, (S == 3 ? 3 : 2)>;  // 128 x 64
template <int S>
using CfgW = ffma::Cfg<64, 128, 2, 2, 8, S, ffma::kLoaderTma, (S == 3 ? 3 : 2)>;  // 64 x 128
template <int S>
using CfgS = ffma::Cfg<32, 128, 1, 4, 4, S, ffma::kLoaderTma, (S == 3 ? 3 : 2)>;  // 32 x 128

constexpr int THREADS = 128;
constexpr int SLOT_BYTES = 24 * 1024;  // 16 KB + 8 KB per 32-deep k block (4 + 16 KB skinny)
static_assert(CfgT<3>::STAGE_BYTES == SLOT_BYTES && CfgW<3>::STAGE_BYTES == SLOT_BYTES &&
                  CfgS<3>::STAGE_BYTES <= SLOT_BYTES && CfgS<3>::THREADS == THREADS,
              "");
enum TileShape { kTileTall = 0, kTileWide = 1, kTileSkinny = 2 };  // 128x64, 64x128, 32x128

inline int tile_bm(int t) { return t == kTileTall ? 128 : t == kTileWide ? 64 : 32; }
inline int tile_bn(int t) { return t == kTileTall ? 64 : 128; }

// Throughput of each tile relative to 128 x 64 on work that fills them
// (measured on a B200 with the single-GEMM kernels of the same shapes).  A
// problem leaves its bucket's tile for another when that tile's zero-padded
// area divided by its efficiency is at least 2% smaller.
inline double tile_efficiency(int t) {
    return t == kTileTall ? 1.0 : t == kTileWide ? 0.994 : 0.75;
}

struct GProblem {
    Operands op;
    int tile;      // a TileShape: the tile of the problem's rows (all of them,
                   // or the bulk when `rem_tile` covers a remainder strip)
    int rem_tile;  // tile of the last rows when they are a strip of their own, else -1
    int rem_m0;    // first row of that strip
    int shapes;    // bit t: the problem has tiles of shape t (a map pair per shape)
    int tma;       // tensor maps valid
    int split;     // k splits
    int kbps;      // k blocks per split
    int depth;     // k blocks kept in flight through the stage ring (2..S)
    int tiles_n;
    int cnt_base;  // first tile ticket (split > 1)
    long long ws_base;  // first workspace float (split > 1)
};

// One work item: a tile of one problem (its shape, its first row and column)
// and one k split.  tl is the tile's index within its problem (split-K
// tickets and partials), used only when the problem is split.
struct GItem {
    int prob, m0, n0, ks;
    int tile, tl;
};

struct GParams {
    const GProblem* probs;
    const GItem* items;
    const CUtensorMap* maps;  // 6 per problem: (A, B) for each tile shape it uses
    float* ws;
    int* counters;  // [0] work ticket, [1..] split-K tile tickets
    int* status;
    int n_items;
};

template <int S>
constexpr int smem_bytes() {
    return S * SLOT_BYTES + 1024;
}

// One work item on the FFMA core.  Returns false (uniformly across the CTA)
// if a bounded wait expired.
template <class C, bool TMA, int S>
__device__ __forceinline__ bool run_item(const GParams& gp, const GProblem& pr, const GItem& it,
                                         int item_prob, uint8_t* smem, uint64_t* full_bar,
                                         uint32_t& g, int* last_s) {
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int wm = warp / C::WN, wn = warp % C::WN;
    int lm, ln;
    ffma::lane_coords(lane, lm, ln);
    const int m0 = it.m0, n0 = it.n0;
    const int nk = (pr.op.k + C::BK - 1) / C::BK;
    const int kb0 = it.ks * pr.kbps;
    const int kb1 = min(nk, kb0 + pr.kbps);
    const int nkb = max(0, kb1 - kb0);

    uint32_t a_base, xa0, xa1;
    ffma::a_coords<C>(wm, lm, a_base, xa0, xa1);
    const uint32_t b_base = static_cast<uint32_t>((wn * 8 * C::TN + ln * 4) * 4);

    float acc[C::TM][C::TN];
#pragma unroll
    for (int i = 0; i < C::TM; ++i)
#pragma unroll
        for (int j = 0; j < C::TN; ++j) acc[i][j] = 0.0f;

    if constexpr (TMA) {
        const CUtensorMap* tmA = gp.maps + 6 * item_prob + 2 * it.tile;
        const CUtensorMap* tmB = tmA + 1;
        int issued = 0;
        auto issue = [&](int j) {
            const uint32_t gs = g + j;
            const int s = gs % S;
            uint8_t* st = smem + s * SLOT_BYTES;
            mbar_arrive_expect_tx(&full_bar[s], C::STAGE_TX);
            tma_load_2d(st, tmA, &full_bar[s], (kb0 + j) * C::BK, m0);
            tma_load_2d(st + C::A_BYTES, tmB, &full_bar[s], n0, (kb0 + j) * C::BK);
        };
        if (tid == 0) {
            const int depth = min(S, pr.depth);  // the bucket's stage count
            // the previous item's generic reads of the ring (ordered by the CTA
            // barrier between items) before these TMA refills
            fence_proxy_async_shared();
            for (; issued < depth && issued < nkb; ++issued) issue(issued);
        }
        for (int j = 0; j < nkb; ++j) {
            const uint32_t gs = g + j;
            const int s = gs % S;
            const bool ok = mbar_wait(&full_bar[s], (gs / S) & 1);
            if (__syncthreads_or(!ok)) {
                if (tid == 0) {
                    atomicExch(gp.status, SGEMM_B200_ERR_TIMEOUT);
                    for (int q = j; q < issued; ++q)
                        if (!mbar_wait(&full_bar[(g + q) % S], ((g + q) / S) & 1)) break;
                }
                return false;
            }
            if (tid == 0 && j > 0 && issued < nkb) {
                fence_proxy_async_shared();  // generic reads of the stage before its TMA refill
                issue(issued++);
            }
            const uint8_t* st = smem + s * SLOT_BYTES;
            ffma::compute_stage<C>(st, st + C::A_BYTES, a_base, xa0, xa1, b_base, acc);
        }
        g += nkb;
    } else {
#pragma unroll
        for (int s = 0; s < S - 1; ++s) {
            if (s < nkb) {
                uint8_t* st = smem + s * SLOT_BYTES;
                ffma::load_stage_async4<C>(pr.op, st, st + C::A_BYTES, m0, n0, (kb0 + s) * C::BK,
                                           tid);
            }
            cp_async_commit();
        }
        for (int j = 0; j < nkb; ++j) {
            cp_async_wait<S - 2>();
            __syncthreads();
            const int nxt = j + S - 1;
            if (nxt < nkb) {
                uint8_t* st = smem + (nxt % S) * SLOT_BYTES;
                ffma::load_stage_async4<C>(pr.op, st, st + C::A_BYTES, m0, n0, (kb0 + nxt) * C::BK,
                                           tid);
            }
            cp_async_commit();
            const uint8_t* st = smem + (j % S) * SLOT_BYTES;
            ffma::compute_stage<C>(st, st + C::A_BYTES, a_base, xa0, xa1, b_base, acc);
        }
        cp_async_wait<0>();
    }

    // epilogue with C read row by row (BATCH 0): batched C loads cost this
    // kernel spills under its register cap
    if (pr.split == 1) {
        ffma::epilogue_any<C, 0>(pr.op, m0, n0, wm, wn, lm, ln, acc, smem);
        return true;
    }

    // ---- split-K: publish the partial, the last split of the tile reduces.
    constexpr int NQ = C::TM * C::TN / 4;
    constexpr int TILE = C::BM * C::BN;
    const int tile_local = it.tl;
    float4* tile_ws = reinterpret_cast<float4*>(gp.ws + pr.ws_base +
                                                (long long)tile_local * pr.split * TILE);
    float4* mine = tile_ws + (long long)it.ks * (TILE / 4);
#pragma unroll
    for (int i = 0; i < C::TM; ++i)
#pragma unroll
        for (int q = 0; q < C::TN / 4; ++q)
            __stcg(&mine[(i * (C::TN / 4) + q) * THREADS + tid],
                   make_float4(acc[i][4 * q], acc[i][4 * q + 1], acc[i][4 * q + 2],
                               acc[i][4 * q + 3]));
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        const int prev = atomicAdd(&gp.counters[1 + pr.cnt_base + tile_local], 1);
        *last_s = prev == pr.split - 1;
    }
    __syncthreads();
    if (*last_s) {
        __threadfence();
        for (int s = 0; s < pr.split; ++s) {
            const float4* part = tile_ws + (long long)s * (TILE / 4);
#pragma unroll
            for (int i = 0; i < C::TM; ++i)
#pragma unroll
                for (int q = 0; q < C::TN / 4; ++q) {
                    const float4 v = __ldcg(&part[(i * (C::TN / 4) + q) * THREADS + tid]);
                    if (s == 0) {
                        acc[i][4 * q] = v.x;
                        acc[i][4 * q + 1] = v.y;
                        acc[i][4 * q + 2] = v.z;
                        acc[i][4 * q + 3] = v.w;
                    } else {
                        acc[i][4 * q] = __fadd_rn(acc[i][4 * q], v.x);
                        acc[i][4 * q + 1] = __fadd_rn(acc[i][4 * q + 1], v.y);
                        acc[i][4 * q + 2] = __fadd_rn(acc[i][4 * q + 2], v.z);
                        acc[i][4 * q + 3] = __fadd_rn(acc[i][4 * q + 3], v.w);
                    }
                }
        }
        (void)NQ;
        ffma::epilogue_any<C, 0>(pr.op, m0, n0, wm, wn, lm, ln, acc, smem);
    }
    return true;
}

template <int S>
__global__ void __launch_bounds__(THREADS, (S == 3 ? 3 : 2)) grouped_kernel(const GParams gp) {
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[S];
    __shared__ int item_s;
    __shared__ int last_s;
    uint8_t* smem = align_smem_1024(smem_raw);
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&full_bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t g = 0;  // k blocks consumed through the TMA ring (phase tracking)
    while (true) {
        if (tid == 0) item_s = atomicAdd(&gp.counters[0], 1);
        __syncthreads();
        const int idx = item_s;
        if (idx >= gp.n_items) break;
        const GItem it = gp.items[idx];
        const GProblem& pr = gp.probs[it.prob];
        bool ok;
        if (it.tile == kTileTall) {
            ok = pr.tma ? run_item<CfgT<S>, true, S>(gp, pr, it, it.prob, smem, full_bar, g, &last_s)
                        : run_item<CfgT<S>, false, S>(gp, pr, it, it.prob, smem, full_bar, g,
                                                      &last_s);
        } else if (it.tile == kTileSkinny) {
            ok = pr.tma ? run_item<CfgS<S>, true, S>(gp, pr, it, it.prob, smem, full_bar, g, &last_s)
                        : run_item<CfgS<S>, false, S>(gp, pr, it, it.prob, smem, full_bar, g,
                                                      &last_s);
        } else {
            ok = pr.tma ? run_item<CfgW<S>, true, S>(gp, pr, it, it.prob, smem, full_bar, g, &last_s)
                        : run_item<CfgW<S>, false, S>(gp, pr, it, it.prob, smem, full_bar, g,
                                                      &last_s);
        }
        if (!ok) break;
        __syncthreads();  // stages and item_s are free for the next item
    }
}

// ------------------------------------------------------------------ host --

struct Choice {
    int tile = kTileTall;
    int split = 1;
    int depth = 4;  // stage count: k blocks in flight (capped by the launch's ring)
};

// Size buckets: M*N class x K class.
constexpr int kMnClasses = 3, kKClasses = 3, kBuckets = kMnClasses * kKClasses;
inline int bucket_of(int m, int n, int k) {
    const double mn = double(m) * n;
    const int a = mn < 256.0 * 256.0 ? 0 : (mn < 1024.0 * 1024.0 ? 1 : 2);
    const int b = k < 512 ? 0 : (k < 2048 ? 1 : 2);
    return a * kKClasses + b;
}

// The tuning table: the launch's ring size (3 stages and 3 CTAs per SM, or 4
// and 2) and, per size bucket, tile shape, split-K and stage count (how many
// of the ring's stages a problem's items keep in flight).
struct Table {
    int stages = 3;
    Choice c[kBuckets];
};

static bool load_table(const char* path, Table* t) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line, dev_name;
    int sms = -1, stages = -1;
    Table out;
    int seen = 0;
    while (std::getline(f, line)) {
        const size_t d = line.find("\"device\"");
        if (d != std::string::npos) {
            const size_t a = line.find('"', line.find(':', d) + 1);
            const size_t b = line.find('"', a + 1);
            if (a != std::string::npos && b != std::string::npos)
                dev_name = line.substr(a + 1, b - a - 1);
        }
        if (line.find("\"sm_count\"") != std::string::npos)
            std::sscanf(line.c_str() + line.find(':') + 1, "%d", &sms);
        // the launch's ring size (bucket lines carry their own "stages")
        if (line.find("\"stages\"") != std::string::npos &&
            line.find("{\"mn\"") == std::string::npos)
            std::sscanf(line.c_str() + line.find(':') + 1, "%d", &stages);
        int mn, kc, tile, split, depth = 4;
        const size_t p = line.find("{\"mn\"");
        if (p != std::string::npos &&
            std::sscanf(line.c_str() + p,
                        "{\"mn\": %d, \"k\": %d, \"tile\": %d, \"split\": %d, \"stages\": %d", &mn,
                        &kc, &tile, &split, &depth) >= 4 &&
            mn >= 0 && mn < kMnClasses && kc >= 0 && kc < kKClasses && tile >= 0 && tile <= 2 &&
            split >= 1 && split <= 16 && depth >= 2 && depth <= 4) {
            out.c[mn * kKClasses + kc].tile = tile;
            out.c[mn * kKClasses + kc].split = split;
            out.c[mn * kKClasses + kc].depth = depth;
            ++seen;
        }
    }
    const DeviceInfo& di = device_info();
    // A table tuned on another GPU model or SM count does not apply here.
    if (dev_name != di.name || sms != di.sm_count) return false;
    if (stages == 3 || stages == 4) out.stages = stages;
    *t = out;
    return seen > 0;
}

static bool save_table(const char* path, const Table& t) {
    std::ofstream f(path);
    if (!f) return false;
    const DeviceInfo& di = device_info();
    f << "{\n \"format\": \"sgemm_b200 grouped tuning v2\",\n";
    f << " \"device\": \"" << di.name << "\",\n";
    f << " \"sm_count\": " << di.sm_count << ",\n";
    f << " \"stages\": " << t.stages << ",\n";
    f << " \"buckets\": [\n";
    for (int a = 0; a < kMnClasses; ++a)
        for (int b = 0; b < kKClasses; ++b) {
            const Choice& ch = t.c[a * kKClasses + b];
            f << "  {\"mn\": " << a << ", \"k\": " << b << ", \"tile\": " << ch.tile
              << ", \"split\": " << ch.split << ", \"stages\": " << ch.depth << "}"
              << (a == kMnClasses - 1 && b == kKClasses - 1 ? "\n" : ",\n");
        }
    f << " ]\n}\n";
    return bool(f);
}

static bool tma_ok(const sgemm_b200_problem& p) {
    return p.k > 0 && (p.lda % 4 == 0) && (p.ldb % 4 == 0) &&
           (reinterpret_cast<uintptr_t>(p.A) % 16 == 0) &&
           (reinterpret_cast<uintptr_t>(p.B) % 16 == 0);
}

}  // namespace grouped
}  // namespace sgb

struct sgemm_b200_grouped_plan {
    int device = -1;
    int stages = 4;
    int n_items = 0;
    int n_tiles = 0;
    int grid = 0;
    size_t ws_floats = 0;
    int n_counters = 0;
    sgb::grouped::GProblem* d_probs = nullptr;
    sgb::grouped::GItem* d_items = nullptr;
    CUtensorMap* d_maps = nullptr;
    float* d_ws = nullptr;
    int* d_counters = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap_stream = nullptr;
};

namespace sgb {
namespace grouped {

static void free_plan(sgemm_b200_grouped_plan* p) {
    if (!p) return;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
    cudaFree(p->d_probs);
    cudaFree(p->d_items);
    cudaFree(p->d_maps);
    cudaFree(p->d_ws);
    cudaFree(p->d_counters);
    delete p;
}

// Host-only part of a plan: per-problem choices and the longest-first item list.
struct Schedule {
    std::vector<GProblem> probs;
    std::vector<GItem> items;
    long long ws_floats = 0;
    int tickets = 0;
    int tiles = 0;
};

static int make_schedule(const sgemm_b200_problem* probs, int count, const Table& table,
                         Schedule* out) {
    if (count < 0 || (count > 0 && !probs)) return SGEMM_B200_ERR_INVALID_ARG;
    for (int i = 0; i < count; ++i) {
        const sgemm_b200_problem& q = probs[i];
        const int s = check_gemm_args(q.m, q.n, q.k, &q.alpha, q.A, q.lda, q.B, q.ldb, &q.beta,
                                      q.C, q.ldc);
        if (s != SGEMM_B200_OK) return s;
    }
    Schedule sc;
    sc.probs.resize(count);
    struct Weighted {
        GItem it;
        double cost;
    };
    std::vector<Weighted> items;
    for (int i = 0; i < count; ++i) {
        const sgemm_b200_problem& q = probs[i];
        GProblem& g = sc.probs[i];
        g.op.m = q.m;
        g.op.n = q.n;
        g.op.k = q.k;
        g.op.lda = q.lda;
        g.op.ldb = q.ldb;
        g.op.ldc = q.ldc;
        g.op.alpha = q.alpha;
        g.op.beta = q.beta;
        g.op.A = q.A;
        g.op.B = q.B;
        g.op.C = q.C;
        g.op.vec_c = (q.ldc % 4 == 0) && (reinterpret_cast<uintptr_t>(q.C) % 16 == 0);
        const Choice ch = table.c[bucket_of(q.m, q.n, q.k)];
        // Padded area per unit efficiency of covering `rows` rows with tile t.
        auto area = [&](int rows, int t) {
            return double(div_up(rows, tile_bm(t)) * tile_bm(t)) *
                   double(div_up(q.n, tile_bn(t)) * tile_bn(t)) / tile_efficiency(t);
        };
        // Problem geometry: a problem a few rows tall (the 32 x 128 tile) or
        // one whose edges fit the other 8 x 8 tile better loses less work to
        // zero padding on that tile.
        int best = ch.tile;
        for (int t : {kTileTall, kTileWide, kTileSkinny})
            if (area(q.m, t) < 0.98 * area(q.m, ch.tile) && area(q.m, t) < area(q.m, best)) best = t;
        g.tile = best;
        g.rem_tile = -1;
        g.rem_m0 = q.m;
        const int nk = div_up(q.k, 32);
        int split = std::max(1, std::min(ch.split, nk));
        g.kbps = nk > 0 ? div_up(nk, split) : 0;
        if (g.kbps > 0) split = div_up(nk, g.kbps);  // no empty splits
        g.split = split;
        g.depth = ch.depth;
        if (split == 1 && q.m > 0 && q.n > 0) {
            // Rows may also be covered by two tiles: the whole tiles of a
            // taller shape, then the leftover rows as a strip of a shorter
            // one (every element still runs its whole k-ordered chain in one
            // item, so the result is the same).  Taken when it pads at least
            // 2% less than the single tile.
            double best_area = area(q.m, best);
            for (int t : {kTileTall, kTileWide})
                for (int u : {kTileWide, kTileSkinny}) {
                    if (tile_bm(u) >= tile_bm(t)) continue;
                    const int bulk = q.m / tile_bm(t) * tile_bm(t);
                    if (bulk == 0 || bulk == q.m) continue;
                    const double a = area(bulk, t) + area(q.m - bulk, u);
                    if (a < 0.98 * best_area) {
                        best_area = a;
                        g.tile = t;
                        g.rem_tile = u;
                        g.rem_m0 = bulk;
                    }
                }
        }
        g.tma = tma_ok(q) ? 1 : 0;
        g.shapes = (1 << g.tile) | (g.rem_tile >= 0 ? 1 << g.rem_tile : 0);
        const int bm = tile_bm(g.tile), bn = tile_bn(g.tile);
        const int tm = q.m > 0 ? div_up(g.rem_m0, bm) : 0;
        const int tn = q.n > 0 ? div_up(q.n, bn) : 0;
        g.tiles_n = tn;
        g.cnt_base = sc.tickets;
        g.ws_base = sc.ws_floats;
        if (split > 1) {
            sc.tickets += tm * tn;
            sc.ws_floats += (long long)tm * tn * split * bm * bn;
        }
        // cost ~ FMAs of the item plus a fixed pipeline fill / epilogue term
        auto add = [&](int tile, int m0, int n0, int tl, int ks) {
            const int kb = std::min(g.kbps, nk - ks * g.kbps);
            const double c = double(tile_bm(tile)) * tile_bn(tile) * (std::max(kb, 0) + 6) * 32;
            items.push_back({GItem{i, m0, n0, ks, tile, tl}, c});
        };
        for (int a = 0; a < tm; ++a)
            for (int b = 0; b < tn; ++b)
                for (int ks = 0; ks < split; ++ks) add(g.tile, a * bm, b * bn, a * tn + b, ks);
        sc.tiles += tm * tn;
        if (g.rem_tile >= 0) {  // the remainder strip (split == 1 only)
            const int rbm = tile_bm(g.rem_tile), rbn = tile_bn(g.rem_tile);
            const int rtm = div_up(q.m - g.rem_m0, rbm), rtn = div_up(q.n, rbn);
            for (int a = 0; a < rtm; ++a)
                for (int b = 0; b < rtn; ++b) add(g.rem_tile, g.rem_m0 + a * rbm, b * rbn, 0, 0);
            sc.tiles += rtm * rtn;
        }
    }
    std::stable_sort(items.begin(), items.end(),
                     [](const Weighted& x, const Weighted& y) { return x.cost > y.cost; });
    sc.items.resize(items.size());
    for (size_t i = 0; i < items.size(); ++i) sc.items[i] = items[i].it;
    *out = std::move(sc);
    return SGEMM_B200_OK;
}

// The tensor maps of one problem: an (A, B) pair for each tile shape it uses,
// at maps[2 * shape] and maps[2 * shape + 1] (six slots per problem).
static bool encode_problem_maps(const GProblem& g, CUtensorMap* maps) {
    for (int t = 0; t < 3; ++t) {
        if (!(g.shapes & (1 << t))) continue;
        if (!encode_tensor_map_2d(&maps[2 * t], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, g.op.A,
                                  (uint64_t)g.op.k, (uint64_t)g.op.m, (uint64_t)g.op.lda * 4, 32,
                                  tile_bm(t), CU_TENSOR_MAP_SWIZZLE_128B) ||
            !encode_tensor_map_2d(&maps[2 * t + 1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, g.op.B,
                                  (uint64_t)g.op.n, (uint64_t)g.op.k, (uint64_t)g.op.ldb * 4,
                                  tile_bn(t), 32, CU_TENSOR_MAP_SWIZZLE_NONE))
            return false;
    }
    return true;
}

// The kernels' dynamic shared-memory attribute, once per device (attributes
// belong to the device's context); a thread that sees the flag also sees the
// attributes set.
static void set_kernel_attributes() {
    static std::atomic<bool> done[64];
    static std::mutex mu;
    const int dev = device_info().device;
    if (dev < 0 || dev >= 64 || done[dev].load(std::memory_order_acquire)) return;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev].load(std::memory_order_relaxed)) return;
    cudaFuncSetAttribute(grouped_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         smem_bytes<3>());
    cudaFuncSetAttribute(grouped_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         smem_bytes<4>());
    done[dev].store(true, std::memory_order_release);
}

// Persistent CTAs per SM of the kernel variant with `stages` stages.
static int resident_per_sm(int stages) {
    int occ = 0;
    const cudaError_t e =
        stages == 3 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, grouped_kernel<3>,
                                                                    THREADS, smem_bytes<3>())
                    : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, grouped_kernel<4>,
                                                                    THREADS, smem_bytes<4>());
    return (e == cudaSuccess && occ > 0) ? occ : 1;
}

static int build_plan(const sgemm_b200_problem* probs, int count, const Table& table,
                      sgemm_b200_grouped_plan** out) {
    if (!out) return SGEMM_B200_ERR_INVALID_ARG;
    Schedule sc;
    int st = make_schedule(probs, count, table, &sc);
    if (st != SGEMM_B200_OK) return st;
    if (!device_is_sm100()) return SGEMM_B200_ERR_UNSUPPORTED;
    auto* plan = new sgemm_b200_grouped_plan();
    plan->device = device_info().device;
    plan->stages = table.stages;
    plan->n_tiles = sc.tiles;
    plan->n_items = (int)sc.items.size();
    plan->ws_floats = (size_t)sc.ws_floats;
    plan->n_counters = 1 + sc.tickets;

    std::vector<CUtensorMap> maps(6 * (size_t)std::max(count, 1));
    std::memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
    for (int i = 0; i < count; ++i) {
        const GProblem& g = sc.probs[i];
        if (g.tma && !encode_problem_maps(g, &maps[6 * (size_t)i])) {
            free_plan(plan);
            return SGEMM_B200_ERR_CUDA;
        }
    }

    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t x) {
        if (e == cudaSuccess) e = x;
    };
    chk(cudaMalloc(&plan->d_probs, sizeof(GProblem) * std::max(count, 1)));
    chk(cudaMalloc(&plan->d_items, sizeof(GItem) * std::max<size_t>(sc.items.size(), 1)));
    chk(cudaMalloc(&plan->d_maps, sizeof(CUtensorMap) * maps.size()));
    chk(cudaMalloc(&plan->d_counters, sizeof(int) * plan->n_counters));
    if (plan->ws_floats) chk(cudaMalloc(&plan->d_ws, sizeof(float) * plan->ws_floats));
    if (e == cudaSuccess && count)
        chk(cudaMemcpy(plan->d_probs, sc.probs.data(), sizeof(GProblem) * count,
                       cudaMemcpyHostToDevice));
    if (e == cudaSuccess && !sc.items.empty())
        chk(cudaMemcpy(plan->d_items, sc.items.data(), sizeof(GItem) * sc.items.size(),
                       cudaMemcpyHostToDevice));
    if (e == cudaSuccess)
        chk(cudaMemcpy(plan->d_maps, maps.data(), sizeof(CUtensorMap) * maps.size(),
                       cudaMemcpyHostToDevice));
    if (e == cudaSuccess) chk(cudaMemset(plan->d_counters, 0, sizeof(int) * plan->n_counters));
    if (e != cudaSuccess) {
        free_plan(plan);
        return cuda_status(e);
    }
    set_kernel_attributes();
    const int sms = device_info().sm_count;
    plan->grid = std::max(1, std::min(sms * resident_per_sm(plan->stages), plan->n_items));
    *out = plan;
    return SGEMM_B200_OK;
}

static int enqueue(sgemm_b200_grouped_plan* plan, cudaStream_t stream) {
    if (plan->n_items == 0) return SGEMM_B200_OK;
    GParams p;
    p.probs = plan->d_probs;
    p.items = plan->d_items;
    p.maps = plan->d_maps;
    p.ws = plan->d_ws;
    p.counters = plan->d_counters;
    p.status = device_status_ptr();
    p.n_items = plan->n_items;
    if (!p.status) return SGEMM_B200_ERR_CUDA;
    cudaError_t e = cudaMemsetAsync(plan->d_counters, 0, sizeof(int) * plan->n_counters, stream);
    if (e != cudaSuccess) return cuda_status(e);
    if (plan->stages == 3)
        grouped_kernel<3><<<plan->grid, THREADS, smem_bytes<3>(), stream>>>(p);
    else
        grouped_kernel<4><<<plan->grid, THREADS, smem_bytes<4>(), stream>>>(p);
    return cuda_status(cudaGetLastError());
}

static int launch(sgemm_b200_grouped_plan* plan, cudaStream_t stream, int use_graph) {
    if (!plan) return SGEMM_B200_ERR_INVALID_ARG;
    if (!use_graph) return enqueue(plan, stream);
    if (!plan->exec) {
        cudaError_t e = cudaSuccess;
        if (!plan->cap_stream) {
            e = cudaStreamCreateWithFlags(&plan->cap_stream, cudaStreamNonBlocking);
            if (e != cudaSuccess) {
                plan->cap_stream = nullptr;
                return cuda_status(e);
            }
        }
        e = cudaStreamBeginCapture(plan->cap_stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_status(e);
        const int s = enqueue(plan, plan->cap_stream);
        cudaGraph_t graph = nullptr;
        e = cudaStreamEndCapture(plan->cap_stream, &graph);
        if (s != SGEMM_B200_OK || e != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            return s != SGEMM_B200_OK ? s : cuda_status(e);
        }
        e = cudaGraphInstantiate(&plan->exec, graph, 0);
        if (e != cudaSuccess) {
            plan->exec = nullptr;
            cudaGraphDestroy(graph);
            return cuda_status(e);
        }
        plan->graph = graph;
    }
    return cuda_status(cudaGraphLaunch(plan->exec, stream));
}

// ------------------------------------------------------------ arena path --
// Batch launcher for the serving loop: device buffers and pinned staging
// buffers are allocated once and grown on demand, so a batch costs a host
// schedule, a few async copies and one kernel launch (no cudaMalloc, no
// graph capture).  An arena must not be reused before its previous batch
// completed (the staging buffers feed async copies).  First allocations are
// generous (min_cap elements), because growing pinned staging means
// cudaFreeHost, which waits for the whole device, in the middle of serving.

template <class T>
static cudaError_t grow(T** d, T** h, size_t* cap, size_t need, cudaStream_t s,
                        size_t min_cap) {
    if (need <= *cap) return cudaSuccess;
    const size_t n = std::max({need, *cap * 2, min_cap});
    if (*d) cudaFreeAsync(*d, s);
    *d = nullptr;
    if (h && *h) {
        cudaFreeHost(*h);
        *h = nullptr;
    }
    cudaMemPool_t pool = library_pool();
    if (!pool) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(d), n * sizeof(T), pool, s);
    if (e == cudaSuccess && h) e = cudaMallocHost(reinterpret_cast<void**>(h), n * sizeof(T));
    if (e == cudaSuccess) *cap = n;
    return e;
}

int arena_launch(Arena* a, const sgemm_b200_problem* probs, int count, cudaStream_t stream) {
    if (!device_is_sm100()) return SGEMM_B200_ERR_UNSUPPORTED;
    Table table;  // built-in choices: split-K off, so results equal the plain path's
    Schedule sc;
    const int st = make_schedule(probs, count, table, &sc);
    if (st != SGEMM_B200_OK) return st;
    if (sc.items.empty()) return SGEMM_B200_OK;
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t x) {
        if (e == cudaSuccess) e = x;
    };
    const size_t n_counters = 1 + (size_t)sc.tickets;
    // first capacities: 256 problems, 64 Ki work items (~1 MB pinned in all)
    chk(grow(&a->d_probs, &a->h_probs, &a->cap_probs, (size_t)count, stream, 256));
    chk(grow(&a->d_items, &a->h_items, &a->cap_items, sc.items.size(), stream, 1 << 16));
    chk(grow(&a->d_maps, &a->h_maps, &a->cap_maps, 6 * (size_t)count, stream, 1536));
    chk(grow<int>(&a->d_counters, nullptr, &a->cap_counters, n_counters, stream, 1024));
    chk(grow<float>(&a->d_ws, nullptr, &a->cap_ws, std::max<size_t>(sc.ws_floats, 1), stream,
                    1));
    if (e != cudaSuccess) return cuda_status(e);
    std::memcpy(a->h_probs, sc.probs.data(), sizeof(GProblem) * count);
    std::memcpy(a->h_items, sc.items.data(), sizeof(GItem) * sc.items.size());
    std::memset(a->h_maps, 0, sizeof(CUtensorMap) * 6 * count);
    for (int i = 0; i < count; ++i) {
        const GProblem& g = sc.probs[i];
        if (g.tma && !encode_problem_maps(g, &a->h_maps[6 * (size_t)i])) return SGEMM_B200_ERR_CUDA;
    }
    chk(cudaMemcpyAsync(a->d_probs, a->h_probs, sizeof(GProblem) * count, cudaMemcpyHostToDevice,
                        stream));
    chk(cudaMemcpyAsync(a->d_items, a->h_items, sizeof(GItem) * sc.items.size(),
                        cudaMemcpyHostToDevice, stream));
    chk(cudaMemcpyAsync(a->d_maps, a->h_maps, sizeof(CUtensorMap) * 6 * count,
                        cudaMemcpyHostToDevice, stream));
    chk(cudaMemsetAsync(a->d_counters, 0, sizeof(int) * n_counters, stream));
    if (e != cudaSuccess) return cuda_status(e);
    set_kernel_attributes();
    GParams p;
    p.probs = a->d_probs;
    p.items = a->d_items;
    p.maps = a->d_maps;
    p.ws = a->d_ws;
    p.counters = a->d_counters;
    p.status = device_status_ptr();
    p.n_items = (int)sc.items.size();
    if (!p.status) return SGEMM_B200_ERR_CUDA;
    static const int per_sm = resident_per_sm(3);  // after the attributes; once, thread-safe
    const int grid = std::max(1, std::min(device_info().sm_count * per_sm, p.n_items));
    grouped_kernel<3><<<grid, THREADS, smem_bytes<3>(), stream>>>(p);
    return cuda_status(cudaGetLastError());
}

void arena_release(Arena* a) {
    cudaFree(a->d_probs);
    cudaFree(a->d_items);
    cudaFree(a->d_maps);
    cudaFree(a->d_counters);
    cudaFree(a->d_ws);
    cudaFreeHost(a->h_probs);
    cudaFreeHost(a->h_items);
    cudaFreeHost(a->h_maps);
    *a = Arena();
}

// Median device time (ms) of `reps` graph launches of a plan.
static double time_plan(sgemm_b200_grouped_plan* plan, cudaStream_t s, int reps) {
    if (launch(plan, s, 1) != SGEMM_B200_OK) return 1e30;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    std::vector<float> t;
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(a, s);
        launch(plan, s, 1);
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        t.push_back(ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
}

}  // namespace grouped
}  // namespace sgb

// ---------------------------------------------------------------- C ABI --

extern "C" int sgemm_b200_grouped_plan_create(sgemm_b200_grouped_plan** plan,
                                              const sgemm_b200_problem* problems, int count,
                                              const char* tuning_json) {
    sgb::grouped::Table t;
    if (tuning_json) sgb::grouped::load_table(tuning_json, &t);  // falls back to defaults
    const int s = sgb::grouped::build_plan(problems, count, t, plan);
    sgb::set_last_status(s);
    return s;
}

extern "C" int sgemm_b200_grouped_plan_launch(sgemm_b200_grouped_plan* plan,
                                              sgemm_b200_stream_t stream, int use_graph) {
    const int s = sgb::grouped::launch(plan, sgb::as_stream(stream), use_graph);
    sgb::set_last_status(s);
    return s;
}

extern "C" int sgemm_b200_grouped_plan_info(const sgemm_b200_grouped_plan* plan, int* tiles,
                                            int* work_items, int* grid_ctas) {
    if (!plan) return SGEMM_B200_ERR_INVALID_ARG;
    if (tiles) *tiles = plan->n_tiles;
    if (work_items) *work_items = plan->n_items;
    if (grid_ctas) *grid_ctas = plan->grid;
    return SGEMM_B200_OK;
}

extern "C" void sgemm_b200_grouped_plan_destroy(sgemm_b200_grouped_plan* plan) {
    sgb::grouped::free_plan(plan);
}

extern "C" int sgemm_b200_grouped(const sgemm_b200_problem* problems, int count,
                                  sgemm_b200_stream_t stream) {
    sgemm_b200_grouped_plan* plan = nullptr;
    int s = sgemm_b200_grouped_plan_create(&plan, problems, count, nullptr);
    if (s != SGEMM_B200_OK) return s;
    s = sgb::grouped::launch(plan, sgb::as_stream(stream), 0);
    // The plan's buffers must outlive the kernel.
    cudaError_t e = cudaStreamSynchronize(sgb::as_stream(stream));
    if (s == SGEMM_B200_OK && e != cudaSuccess) s = sgb::cuda_status(e);
    sgb::grouped::free_plan(plan);
    sgb::set_last_status(s);
    return s;
}

extern "C" int sgemm_b200_grouped_sequential(const sgemm_b200_problem* problems, int count,
                                             sgemm_b200_stream_t stream) {
    if (count < 0 || (count > 0 && !problems)) return SGEMM_B200_ERR_INVALID_ARG;
    for (int i = 0; i < count; ++i) {
        const sgemm_b200_problem& q = problems[i];
        const int s = sgemm_b200(q.m, q.n, q.k, &q.alpha, q.A, q.lda, q.B, q.ldb, &q.beta, q.C,
                                 q.ldc, stream);
        if (s != SGEMM_B200_OK) return s;
    }
    return SGEMM_B200_OK;
}

extern "C" int sgemm_b200_grouped_schedule(const sgemm_b200_problem* problems, int count,
                                           const char* tuning_json, int* tiles, int* work_items,
                                           size_t* workspace_bytes) {
    sgb::grouped::Table t;
    if (tuning_json) sgb::grouped::load_table(tuning_json, &t);
    sgb::grouped::Schedule sc;
    const int s = sgb::grouped::make_schedule(problems, count, t, &sc);
    if (s != SGEMM_B200_OK) return s;
    if (tiles) *tiles = sc.tiles;
    if (work_items) *work_items = (int)sc.items.size();
    if (workspace_bytes) *workspace_bytes = (size_t)sc.ws_floats * sizeof(float);
    return SGEMM_B200_OK;
}

extern "C" int sgemm_b200_grouped_bucket(int m, int n, int k) {
    return sgb::grouped::bucket_of(m, n, k);
}

extern "C" int sgemm_b200_autotune_grouped(const sgemm_b200_problem* problems, int count,
                                           const char* json_path) {
    using namespace sgb::grouped;
    if (!json_path) return SGEMM_B200_ERR_INVALID_ARG;
    if (!sgb::device_is_sm100()) return SGEMM_B200_ERR_UNSUPPORTED;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
        return SGEMM_B200_ERR_CUDA;
    bool present[kBuckets] = {false};
    for (int i = 0; i < count; ++i)
        present[bucket_of(problems[i].m, problems[i].n, problems[i].k)] = true;
    Table best;
    auto measure = [&](const Table& t) {
        sgemm_b200_grouped_plan* plan = nullptr;
        if (build_plan(problems, count, t, &plan) != SGEMM_B200_OK) return 1e30;
        const double ms = time_plan(plan, s, 5);
        free_plan(plan);
        return ms;
    };
    double best_ms = measure(best);
    // The launch's ring size, then per bucket present in the workload (by
    // coordinate descent): tile shape x split-K, then the bucket's stage count.
    // A candidate must win by 1% to replace the current choice.
    for (int st : {3, 4}) {
        if (st == best.stages) continue;
        Table t = best;
        t.stages = st;
        const double ms = measure(t);
        if (ms < best_ms) {
            best_ms = ms;
            best = t;
        }
    }
    auto consider = [&](const Table& t) {
        const double ms = measure(t);
        if (ms < best_ms * 0.99) {
            best_ms = ms;
            best = t;
        }
    };
    for (int b = 0; b < kBuckets; ++b) {
        if (!present[b]) continue;
        const int kclass = b % kKClasses, mnclass = b / kKClasses;
        for (int tile : {kTileTall, kTileWide, kTileSkinny}) {
            if (tile == kTileSkinny && mnclass == 2) continue;  // large problems: no
            for (int split : {1, 2, 4, 8, 16}) {
                if (split > 1 && kclass == 0) continue;  // short K: nothing to split
                Table t = best;
                t.c[b].tile = tile;
                t.c[b].split = split;
                if (t.c[b].tile == best.c[b].tile && t.c[b].split == best.c[b].split) continue;
                consider(t);
            }
        }
        for (int depth : {2, 3, 4}) {
            if (depth == best.c[b].depth) continue;
            Table t = best;
            t.c[b].depth = depth;
            consider(t);
        }
    }
    cudaStreamDestroy(s);
    return save_table(json_path, best) ? SGEMM_B200_OK : SGEMM_B200_ERR_INVALID_ARG;
}
