// surrogate.cuh -- the learned bond-order potential: shapes, parameter
// layout and the device workspace shared by the inference and training
// kernels.  Not part of the public C-ABI.
//
// Row = directed bond (i -> j) of the REBO list with r_ij <= 2.0.  Each row
// carries a 32-wide descriptor of i's other bonds as seen from i -> j; a
// 3 x 128 SiLU network maps it to the bond order b_ij, and its gradient
// network gives db_ij/dx.  The REBO pair functions and the reference's force
// construction (AI:325-418) turn b and db/dr_k into energy, forces and virial.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "fmd_internal.h"

namespace fmd {
namespace sg {

constexpr int D = 32;        // descriptor width (4 radial x 8 angular, last = bias unit)
constexpr int H = 128;       // hidden width (column 127 = bias unit)
constexpr int NR = 4, NA = 8;
constexpr int TILE = 128;    // rows per tensor-core tile
constexpr double RHO_C = 1.55, RHO_W = 0.45;   // rho(r) = (r - 1.55) / 0.45

// FP64 master parameter vector: W1[D][H] W2[H][H] W3[H][H] w4[H] m[D] s[D] b0 bs
constexpr int OW1 = 0, OW2 = OW1 + D * H, OW3 = OW2 + H * H, OW4 = OW3 + H * H;
constexpr int OM = OW4 + H, OS = OM + D, OB0 = OS + D, OBS = OB0 + 1, NPARAM = OBS + 1;

// BF16 weight images in the interleaved operand layout (umma.cuh):
// W1 as 128 rows (out) x 32 columns (in), W2 and W3 as 128 x 128.
constexpr int IMG_W1 = 0, IMG_W2 = IMG_W1 + H * D, IMG_W3 = IMG_W2 + H * H, IMG_N = IMG_W3 + H * H;
// FP32 vectors: w4[H] m[D] sinv[D] b0 bs
constexpr int V_W4 = 0, V_M = V_W4 + H, V_SINV = V_M + D, V_B0 = V_SINV + D, V_BS = V_B0 + 1, V_N = V_BS + 1;

constexpr int kRowBlocks = kSMs * 8;   // grid of the per-row kernels (grid-stride)

struct Work {
    int na_cap = 0, r_cap = 0, cap = 0;
    int na_used = 0;          // na of the last build_rows (rows = aoff[na_used])
    int* acnt = nullptr;      // [na] rows per atom
    int* aoff = nullptr;      // [na + 1] exclusive scan; aoff[na] = rows
    int* row_i = nullptr;     // [r_cap]
    int* row_s = nullptr;     // [r_cap] list slot of j in i's row
    int* rowid = nullptr;     // [na * cap] row of (i, slot) or -1
    int* partner = nullptr;   // [r_cap] row of (j -> i)
    uint16_t* X = nullptr;    // [r_cap * D] bf16 descriptor tiles (interleaved layout)
    float* b = nullptr;       // [r_cap]
    float* gx = nullptr;      // [r_cap * D] db/dx_n
    double* part = nullptr;   // per-block {E, W9}
    int* err = nullptr;       // [4] kernel status words
    int* bsum = nullptr;      // [na / 256 + 1] rows per block of 256 atoms
    int* boff = nullptr;      // [na / 256 + 2] their exclusive scan
};

cudaError_t work_alloc(Work& w, int na, int cap);
void work_free(Work& w);

// Packs the FP64 master parameters into the BF16 images and FP32 vectors.
cudaError_t pack_params(const double* P, uint16_t* img, float* vec, cudaStream_t st);

// Rows, descriptors, network, forces: F += REBO(learned b), part = per-block
// {E, W9} (kRowBlocks records).  hh = {h, hi} on the device.  A non-null
// gate (device int) that is set makes the pass produce no rows: F is left
// alone and the partials are zero.
cudaError_t rebo_forces(Work& w, const uint16_t* img, const float* vec, const double* pos, const double* hh,
                        const int* cnt, const int* list, int cap, int na, double* F, double* part,
                        cudaStream_t st, const int* gate = nullptr);
// The stages of rebo_forces, for tests and training.
cudaError_t build_rows(Work& w, const float* vec, const double* pos, const double* hh, const int* cnt,
                       const int* list, int cap, int na, cudaStream_t st, const int* gate = nullptr);
cudaError_t run_mlp(Work& w, const uint16_t* img, const float* vec, cudaStream_t st);
cudaError_t assemble(Work& w, const float* vec, const double* pos, const double* hh, const int* cnt,
                     const int* list, int cap, int na, double* F, double* part, cudaStream_t st);

}  // namespace sg
}  // namespace fmd
