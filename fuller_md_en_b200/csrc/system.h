// system.h -- host-side owner of one device-resident system.
#pragma once
#include <vector>
#include "step.h"

namespace fmd {

constexpr int kInCap = 1024;   // incoming (transposed) LJ entries per atom

struct System {
    fmd_ctx* ctx = nullptr;
    fmd_run_params p{};
    StepParams sp{};
    StepArrays arr{};
    CellList cells_a, cells_b;
    double rc_a = 0, rc2_a = 0, rc_b = 0, rc2_b = 0;
    double h0[9] = {0};
    int* dropped = nullptr;            // device: {list a, list b} overflow counts
    bool initialized = false;
    cudaGraphExec_t graphs[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    std::vector<void*> owned;

    template <class T> cudaError_t alloc(T** p, size_t count, const T* src);
    int alloc_common(const double* pos, const double* vel, const double* h, const fmd_npt* npt);
    int alloc_lists(double rc_list_a, int cap_a, double rc_list_b, int cap_b, bool transpose);
    int upload_topology(const fmd_mm_topology* t);
    cudaError_t enqueue_rebuild(cudaStream_t st);
    cudaError_t enqueue_variant(bool rebuild, bool phase, cudaStream_t st);
    cudaError_t enqueue_one(int g, cudaStream_t st);
    int init();
    int capture(bool rebuild, bool phase);
    int run(int first, int last, fmd_obs* obs);
    int enqueue(int first, int last);
    int nonfinite_check();
    void release();
    ~System() { release(); }
};

}  // namespace fmd
