// ljprune.h -- dynamic pruning of the LJ gather's full rows (ljprune.cu).
// Not part of the public C-ABI.
#pragma once
#include <cuda_runtime.h>

#include "kernels.h"

namespace fmd {

// Device state of the pruned LJ rows of one system: after a list build, and
// whenever the motion since the last prune could have brought a dropped entry
// inside the cutoff, the gather walks the full rows and writes the entries
// within rc + delta (in row order); other steps walk those shorter rows.
struct LJPrune {
    bool ok = false;
    double delta = 0.0;           // buffer beyond the cutoff (A); 0: pruning off
    int n = 0, stride = 0;        // atoms, row stride (the full rows' in_cap)
    double rc = 0.0;              // LJ cutoff of the system's force field
    int* cnt = nullptr;           // [n] pruned row lengths
    int* list = nullptr;          // [n * stride] pruned rows
    double* sb = nullptr;         // [3 n] fractional positions at the last prune
    double* hb = nullptr;         // [9] cell at the last prune
    unsigned long long* words = nullptr;  // [1] bits of the largest displacement since the last prune
    unsigned long long* stats = nullptr;  // [2] {force evaluations, prune evaluations}
};

// Displacement bound that forces the next evaluation to prune (~1.4e306 A).
constexpr unsigned long long kPruneMark = 0x7F7F7F7F7F7F7F7Full;

// Clears the counters, snapshot and cell on st and marks the first
// evaluation as a prune (the arrays are owned by the system; the row buffer
// is written by that prune before any read).
cudaError_t lj_prune_clear(const LJPrune& p, cudaStream_t st);
// After a list build (and at set-up): the next evaluation prunes.
cudaError_t lj_prune_mark(const LJPrune& p, cudaStream_t st);
// Output and decision block of the gather (lj_gather_launch's po).
LJPruneOut lj_prune_out(const LJPrune& p);

}  // namespace fmd
