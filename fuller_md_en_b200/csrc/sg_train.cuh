// sg_train.cuh -- training workspace and launch interface of the learned
// bond-order potential.  Not part of the public C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "surrogate.cuh"

namespace fmd {
namespace sg {

// BF16 operand tiles (interleaved layout, 128 rows x 128 columns per row tile)
// written by the chain kernel and read by the weight-gradient kernel.
struct OperandTiles {
    uint16_t *h1 = nullptr, *h2 = nullptr, *g1 = nullptr, *g2 = nullptr, *g3 = nullptr;
    uint16_t *tb1 = nullptr, *tb2 = nullptr, *z1 = nullptr, *z2 = nullptr, *z3 = nullptr;
};

struct TrainWork {
    int r_cap = 0, na_cap = 0;
    OperandTiles t;
    uint16_t* U = nullptr;   // [r_cap * D] dL/d(db/dxn) tiles
    float* beta = nullptr;   // [r_cap] dL/db
    double* lamF = nullptr;  // [3 * na] dL/dF
    double* part = nullptr;  // [kRowBlocks]
    double* sc = nullptr;    // [32] scalars: E,W9 | sum dF^2 | lambda_E, lambda_W9
};

struct AdamArgs {
    double lr, b1, b2, eps, bc1, bc2, scale, clip;
};

// Gradient buffer (FP32): dW1^T [H][D] | dW2^T [H][H] | dW3^T [H][H] | dw4 [H]
constexpr int GRAD_N = H * D + 2 * H * H + H;

cudaError_t train_alloc(TrainWork& tw, const Work& w);
void train_free(TrainWork& tw);

// Adds the loss gradient of one snapshot to grad and {loss, mean dF^2} to
// loss_acc[0..1].  ref10 = {E_ref, W_ref[9]} on the device; F is scratch [3na].
cudaError_t accumulate_grad(Work& w, TrainWork& tw, const uint16_t* img, const float* vec, const double* pos,
                            const double* hh, const int* cnt, const int* list, int cap, int na, const double* Fref,
                            const double* ref10, double wE, double wF, double wW, double* F, double* loss_acc,
                            float* grad, cudaStream_t st);
// Adam on the network weights of the FP64 master vector, then repack.
cudaError_t adam_step(double* P, double* m, double* v, const float* grad, const AdamArgs& a, uint16_t* img,
                      float* vec, cudaStream_t st);
// out[0] += mean over the 3na components of (F - Fref)^2 (part: kRowBlocks doubles).
cudaError_t force_mse(const double* F, const double* Fref, int na, double* part, double* out, cudaStream_t st);
// acc[2f] += sum of descriptor f over the rows of the last build_rows, acc[2f+1] += sum of squares.
cudaError_t feature_sums(const Work& w, double* acc, cudaStream_t st);
// Gradient buffer -> master parameter layout (FP64, zeros for m, s, b0, bs).
cudaError_t grad_to_params(const float* grad, double scale, double* out, cudaStream_t st);

}  // namespace sg
}  // namespace fmd
