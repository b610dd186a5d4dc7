// system.h -- host-side owner of one device-resident system.
#pragma once
#include <memory>
#include <vector>
#include "ljprune.h"
#include "molnlist.h"
#include "sg_host.h"
#include "step.h"

namespace fmd {

constexpr int kInCap = 1024;   // incoming (transposed) LJ entries per atom; full rows add the own row
constexpr double kPruneDelta = 0.5;   // default buffer of the pruned LJ rows beyond the cutoff (A)

struct System {
    fmd_ctx* ctx = nullptr;
    fmd_run_params p{};
    StepParams sp{};
    StepArrays arr{};
    CellList cells_a, cells_b;
    MolLists mol;                      // molecule-wise list builder (contiguous molecules)
    LJPrune prune;                     // pruned LJ rows (AIREBO, MM; prune.ok false: full rows only)
    double rc_a = 0, rc2_a = 0, rc_b = 0, rc2_b = 0;
    double h0[9] = {0};
    int* dropped = nullptr;            // device: {list a, list b} overflow counts
    int* rebo_bsum = nullptr;          // device scratch of the REBO slot index build
    cudaStream_t side = nullptr;       // captures the rebuild fallback's conditional body
    cudaEvent_t obs_ev[2] = {};        // fmd_system_enqueue_obs: copies of odd / even last steps
    bool initialized = false;
    // one graph per {rebuild, cold/warm phase, judge of the learned REBO term}
    cudaGraphExec_t graphs[2][2][2] = {};
    std::vector<std::pair<void*, size_t>> owned;   // blocks from the context's cache, with their sizes
    std::unique_ptr<SgStep> sg;        // learned REBO term (AIREBO only), nullptr: plain

    template <class T> cudaError_t alloc(T** p, size_t count, const T* src);
    // DevAlloc hook: untyped blocks owned (and released) like alloc's
    static cudaError_t alloc_raw(void* self, void** p, size_t bytes);
    DevAlloc owned_alloc() { return DevAlloc{this, &System::alloc_raw}; }
    int alloc_common(const double* pos, const double* vel, const double* h, const fmd_npt* npt);
    int alloc_lists(double rc_list_a, int cap_a, double rc_list_b, int cap_b, bool transpose);
    int alloc_prune(double rc_lj);
    int upload_topology(const fmd_mm_topology* t);
    int upload_topology_arrays(const fmd_mm_topology* t);
    // One molecule's topology t (indices within the molecule) replicated on
    // the device over nmol contiguous molecules of natom atoms.
    int replicate_topology(const fmd_mm_topology* t, int nmol, int natom);
    cudaError_t enqueue_rebuild(cudaStream_t st);
    // The cell-grid half rows and their transpose, gated off on the device
    // when the molecule path built this rebuild (the fallback part of
    // enqueue_rebuild for systems whose full rows come from the candidate
    // bitmaps; replica batches run it inside a conditional graph node).
    cudaError_t enqueue_rebuild_fallback(cudaStream_t st);
    // While st is being captured: the fallback as a conditional node that the
    // molecule path's decision switches on only when it rejected this rebuild.
    cudaError_t enqueue_fallback_conditional(cudaStream_t st);
    cudaError_t enqueue_variant(bool rebuild, bool phase, cudaStream_t st, bool judge = false);
    cudaError_t enqueue_one(int g, cudaStream_t st);
    bool judge_step(int g) const { return arr.sg && arr.sg->judge_every > 0 && g % arr.sg->judge_every == 0; }
    int init();
    int tune_lj();
    int tune_lj_pruned(bool run_tuner, bool* pending);
    LJShape pick_lj_shape(bool pruned, int& rc);
    void set_lj_blocks();
    int tune_rigid();
    int capture(bool rebuild, bool phase, bool judge = false);
    void drop_graphs();
    int use_surrogate(fmd_sg* model, int judge_every, double rmse_max);
    int run(int first, int last, fmd_obs* obs);
    int enqueue(int first, int last);
    int nonfinite_check();
    void release();
    ~System() { release(); }
};

}  // namespace fmd

// The C-ABI handle of a system (include/fullermd.h).
struct fmd_system {
    std::unique_ptr<fmd::System> sys;
};
