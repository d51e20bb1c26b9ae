// grouped.h — internal interface of the grouped kernel's batch launcher, used
// by the serving loop.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/sgemm_b200.h"

namespace sgb {
namespace grouped {

struct GProblem;
struct GItem;

// Reusable device + pinned staging buffers for back-to-back grouped launches.
struct Arena {
    GProblem* d_probs = nullptr;
    GItem* d_items = nullptr;
    CUtensorMap* d_maps = nullptr;
    int* d_counters = nullptr;
    float* d_ws = nullptr;
    GProblem* h_probs = nullptr;
    GItem* h_items = nullptr;
    CUtensorMap* h_maps = nullptr;
    size_t cap_probs = 0, cap_items = 0, cap_maps = 0, cap_counters = 0, cap_ws = 0;
};

// Schedule `count` problems (built-in choices, no split-K) and launch one
// persistent grouped kernel on `stream` using the arena's buffers.
int arena_launch(Arena* arena, const sgemm_b200_problem* problems, int count,
                 cudaStream_t stream);
void arena_release(Arena* arena);

}  // namespace grouped
}  // namespace sgb
