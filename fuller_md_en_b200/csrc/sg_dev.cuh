// sg_dev.cuh -- device helpers shared by the inference (surrogate.cu) and
// training (sg_train.cu) kernels of the learned bond-order potential.
#pragma once
#include <cuda_bf16.h>

#include "rebo_fn.cuh"
#include "surrogate.cuh"
#include "umma.cuh"

namespace fmd {
namespace sg {
namespace dev {

using namespace rebo;

// Chebyshev T_0..T_{n-1}(x) and derivatives.
template <int N>
__device__ __forceinline__ void cheb(float x, float* T, float* dT) {
    T[0] = 1.f; dT[0] = 0.f;
    if (N > 1) { T[1] = x; dT[1] = 1.f; }
#pragma unroll
    for (int n = 2; n < N; n++) {
        T[n] = 2.f * x * T[n - 1] - T[n - 2];
        dT[n] = 2.f * T[n - 1] + 2.f * x * dT[n - 1] - dT[n - 2];
    }
}

// A bond is a row when r_ij <= 2.0 and the reference does not skip it
// (AI:292-296: rij > Dmax, or fc < 1e-15 with dfc == 0).
__device__ __forceinline__ bool bond_kept(double r) {
    if (r > DMAX_CC) return false;
    return !(sw_fc(r) < 1e-15 && sw_dfc(r) == 0.0);
}

// Logistic sigmoid by the fast exponential and fast reciprocal (a few ulp;
// every use rounds to BF16 or enters an FP32 sum): 1 / (1 + e^-z).  For
// z < ~-88, e^-z is infinite and the quotient 0.
__device__ __forceinline__ float sigm(float z) { return __fdividef(1.f, 1.f + __expf(-z)); }


// SiLU'(z) and SiLU''(z) from s = sigmoid(z).
__device__ __forceinline__ float dsilu(float z, float s) { return s * (1.f + z * (1.f - s)); }
__device__ __forceinline__ float d2silu(float z, float s) { return s * (1.f - s) * (2.f + z * (1.f - 2.f * s)); }

// 16 consecutive values of row q, columns [col, col+16), of a 128-column
// BF16 tile in the interleaved layout (shared or global memory).
__device__ __forceinline__ void st_tile16(unsigned char* base, int q, int col, const float* v) {
#pragma unroll
    for (int h8 = 0; h8 < 2; h8++) {
        uint4 o;
        o.x = umma::pack_bf16(v[8 * h8 + 0], v[8 * h8 + 1]);
        o.y = umma::pack_bf16(v[8 * h8 + 2], v[8 * h8 + 3]);
        o.z = umma::pack_bf16(v[8 * h8 + 4], v[8 * h8 + 5]);
        o.w = umma::pack_bf16(v[8 * h8 + 6], v[8 * h8 + 7]);
        *reinterpret_cast<uint4*>(base + umma::il_off(q, col + 8 * h8, H)) = o;
    }
}
__device__ __forceinline__ void ld_tile16(const unsigned char* base, int q, int col, float* v) {
#pragma unroll
    for (int h8 = 0; h8 < 2; h8++) {
        const uint4 o = *reinterpret_cast<const uint4*>(base + umma::il_off(q, col + 8 * h8, H));
        const uint32_t w[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
        for (int e = 0; e < 4; e++) {
            v[8 * h8 + 2 * e] = __uint_as_float(w[e] << 16);
            v[8 * h8 + 2 * e + 1] = __uint_as_float(w[e] & 0xFFFF0000u);
        }
    }
}

// Block-wide hand-off from the epilogue threads to the MMA-issuing thread.
__device__ __forceinline__ void to_mma() {
    umma::fence_smem_async();
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
}
// The same hand-off, also returning whether `ok` holds in every thread.
__device__ __forceinline__ bool to_mma_and(bool ok) {
    umma::fence_smem_async();
    umma::fence_before();
    const bool all = __syncthreads_and(ok) != 0;
    umma::fence_after();
    return all;
}

__device__ __forceinline__ void issue(uint32_t d, uint32_t a_base, int a_cols, bool a_mn, uint32_t b_base,
                                      int b_cols, bool b_mn, int N, int ksteps, uint64_t* mbar) {
    const uint32_t id = umma::idesc_bf16(128, N, a_mn, b_mn);
    for (int s = 0; s < ksteps; s++) {
        const uint64_t da = a_mn ? umma::desc_mn(a_base, a_cols, s) : umma::desc_k(a_base, a_cols, s);
        const uint64_t db = b_mn ? umma::desc_mn(b_base, b_cols, s) : umma::desc_k(b_base, b_cols, s);
        umma::mma_bf16(d, da, db, id, s > 0);
    }
    umma::commit(mbar);
}

}  // namespace dev
}  // namespace sg
}  // namespace fmd
