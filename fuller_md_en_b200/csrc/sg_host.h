// sg_host.h -- internal hooks between the learned-potential C-ABI and the
// device-resident systems.  Not part of the public C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "fmd_internal.h"
#include "surrogate.cuh"

struct fmd_sg_data;
struct fmd_sg;

namespace fmd {

struct StepArrays;

// Adds a snapshot whose positions, {h, hi} and REBO list are device arrays;
// its reference REBO energy, forces and virial come from the plain kernel.
int sg_data_add_device(fmd_sg_data* d, const double* pos, const double* hh, const int* cnt, const int* list, int cap,
                       int na, cudaStream_t st);

// Device images of a model's parameters (owned by the model; their addresses
// are fixed for its lifetime, fmd_sg_set_params rewrites them in place).
void sg_model_images(const fmd_sg* m, const uint16_t** img, const float** vec);

// The learned REBO term of one AIREBO system.  Buffers are owned by the
// system and sized for its atom count and REBO list width at attach time.
struct SgStep {
    const uint16_t* img = nullptr;   // model images
    const float* vec = nullptr;
    sg::Work work;                   // rows, descriptors, network outputs
    double* Fj = nullptr;            // [3n] plain REBO forces of a judge step
    double* part_j = nullptr;        // [kRowBlocks * kNV] plain REBO partials of a judge step
    int judge_every = 0;             // judge on global steps divisible by this (0: never)
    double rmse_max = 0.0;           // takeover threshold, eV/A
};

// REBO term of one step into a.Facc / a.part_f1 (sg::kRowBlocks records):
// the learned term while S->sg_off == 0, the plain kernel after a takeover.
// judge: the plain kernel also runs into Fj / part_j, the force RMSE between
// the two is recorded in S, and above rmse_max the plain result replaces the
// learned one and S->sg_off is set for the rest of the run.
cudaError_t sg_enqueue_rebo(SgStep& g, const StepArrays& a, bool judge, cudaStream_t st);

}  // namespace fmd
