// molnlist.h -- neighbour lists of atomistic systems built molecule by
// molecule (molnlist.cu).  Not part of the public C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "fmd_internal.h"
#include "kernels.h"

namespace fmd {

constexpr int kMolPartners = 256;   // partner molecules per molecule (table width)

struct MolLists {
    bool ok = false;          // molecules are contiguous index ranges
    int n = 0, M = 0, pmax = 0;
    int max_atoms = 0;        // atoms of the largest molecule
    int usize = 0;            // atoms of every molecule when all have the same count, else 0
    bool ext = false;         // arrays from a DevAlloc hook (owned elsewhere)
    bool masks = false;       // 32 <= usize <= 64: the full LJ rows come from the candidate bitmaps
    int words = 0;            // bitmap words per atom: 2 pmax (two per higher partner)
    unsigned* bm = nullptr;   // [M * words * usize] kept-candidate bitmaps of the half-row walk
    int* rev = nullptr;       // [M * pmax] position of B among the higher partners of its q-th (lower) partner
    int* off = nullptr;       // [M + 1] first atom of each molecule
    int* amol = nullptr;      // [n] molecule of each atom
    double* cen = nullptr;    // [3 M] centres
    double* rad = nullptr;    // [M] radii
    float4* pos32 = nullptr;  // [n] positions of the build rounded to FP32 (w unused), for the prefilter
    int* npart = nullptr;     // [M] partner count
    int* part = nullptr;      // [M * pmax] partners, ascending
    int* flag = nullptr;      // [2] {molecule path valid, partner overflow}
};

// Host set-up from the atoms' molecule ids; m.ok stays false (the cell-grid
// builder is used) unless every molecule is one contiguous index range.
cudaError_t mol_lists_alloc(MolLists& m, int n, const int* mol_id_host, const DevAlloc& da = DevAlloc{});
void mol_lists_free(MolLists& m);
// Centres, radii and partner molecules for list radius rc; sets flag[0].
cudaError_t mol_partners(MolLists& m, const double* pos, const double* hh, double rc, cudaStream_t st);
// Intramolecular rows (always valid for contiguous molecules).
cudaError_t mol_rows_intra(const MolLists& m, const double* pos, const double* hh, double rc2, int cap, int* cnt,
                           int* list, int* dropped, cudaStream_t st);
// Half-list rows (the reference's truncation at cap); no-ops unless flag[0] is set.
cudaError_t mol_rows_half(const MolLists& m, const double* pos, const double* hh, double rc2, int cap, int* cnt,
                          int* list, int* dropped, cudaStream_t st);
// The LJ gather's full rows (incoming entries ascending, then the row) from
// the candidate bitmaps of the last mol_rows_half (m.masks only); no-op
// unless flag[0] is set.
cudaError_t mol_rows_incoming(const MolLists& m, int cap, const int* cnt, const int* list, int* in_cnt,
                              int* in_list, int in_cap, DevErr* err, cudaStream_t st);

// One replica of a batched molecule-path rebuild (replica batches of MM
// systems, batch.cu): its molecule tables and the lists it builds.
struct MolRep {
    MolLists m;
    const double* pos = nullptr;
    double* hh = nullptr;                 // h then h^-1 (h^-1 recomputed first)
    double rc = 0.0, rc2 = 0.0;           // list radius, squared
    int cap = 0, in_cap = 0;
    int* cnt = nullptr;
    int* list = nullptr;
    int* dropped = nullptr;
    int* in_cnt = nullptr;
    int* in_list = nullptr;
    DevErr* err = nullptr;
    unsigned long long* prune_words = nullptr;   // the replica's pruned-row bound (marked stale), or null
};
// Device table of the replicas and the block offsets (R + 1 each) of the
// batched launches: warp-per-molecule kernels, half rows, full rows.
struct MolBatch {
    const MolRep* reps = nullptr;
    int R = 0;
    const int* off_w = nullptr;
    const int* off_rows = nullptr;
    const int* off_in = nullptr;
    int nblk_w = 0, nblk_rows = 0, nblk_in = 0;
};
// The molecule-path rebuild of every replica of a batch, one launch per
// phase, for equal molecules of 32-64 atoms (the candidate-bitmap path).
// First part: h^-1, centres and radii, partner tables and the path decision
// of each replica; `cond` (a conditional node's handle in the graph being
// captured) is set to 1 when some replica's molecule path is rejected for
// this build, whose cell-grid fallback the caller places next.  Second part:
// the half rows and the gather's full rows of every accepted replica.
cudaError_t mol_rebuild_batch_pre(const MolBatch& b, cudaGraphConditionalHandle cond, cudaStream_t st,
                                  const char** stage = nullptr);
cudaError_t mol_rebuild_batch_rows(const MolBatch& b, cudaStream_t st);

}  // namespace fmd
