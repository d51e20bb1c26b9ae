// split.h — internal interface of the grouped split-precision launcher, used
// by the serving loop.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/sgemm_b200.h"

namespace sgb {
namespace split {

// Reusable device table and pinned staging for back-to-back grouped split
// launches (one per serving slot).  An arena must not be reused before its
// previous launch completed: the launch reads the staging (async copy) and
// the device table (kernels).
struct Arena {
    uint8_t* d = nullptr;  // device table, from the library pool
    uint8_t* h = nullptr;  // pinned staging
    size_t cap = 0;
};

// Workspace bytes one problem needs in a grouped split launch (the same as
// sgemm_b200_split_workspace_size; 0 for k == 0 or an empty C).
size_t problem_workspace_bytes(int path, int m, int n, int k);

// All `count` problems as one grouped pre-pass and one persistent tcgen05
// launch on `stream`; problem i writes its planes to ws[i] (at least
// problem_workspace_bytes bytes, any alignment).  Problems with k == 0 run on
// the plain path (C := beta*C).  Results equal sgemm_b200_split's, bit for bit.
int grouped_launch(Arena* arena, int path, const sgemm_b200_problem* problems,
                   void* const* ws, int count, cudaStream_t stream);
void arena_release(Arena* arena);

}  // namespace split
}  // namespace sgb
