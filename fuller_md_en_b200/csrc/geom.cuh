// geom.cuh -- device geometry primitives shared by all kernels.
//
// Every operation that feeds a discrete decision (neighbour-list membership,
// cutoff tests, image choice) is written with explicit round-to-nearest
// intrinsics so nvcc cannot contract it into FMAs.  The result is bitwise
// the same as the reference built by g++ -O3 for x86-64 (SSE2, no FMA), which
// is what makes the neighbour sets bit-exact.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace fmd {

constexpr double kConv = 9.64853321e-3;     // eV fs^2 / (amu A^2)       (LJ:101)
constexpr double kKB = 8.617333262e-5;      // eV/K                      (LJ:101)
constexpr double kEV2GPa = 160.21766208;    // eV/A^3 -> GPa             (LJ:102)
constexpr double kPi = 3.14159265358979323846;
constexpr unsigned kFull = 0xffffffffu;

// a*x + b*y + c*z evaluated left to right without contraction.
__device__ __forceinline__ double dot3_rn(double a, double b, double c, double x, double y, double z) {
    return __dadd_rn(__dadd_rn(__dmul_rn(a, x), __dmul_rn(b, y)), __dmul_rn(c, z));
}
__device__ __forceinline__ double norm2_rn(double x, double y, double z) {
    return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

// Minimum image as the reference chooses it: round() of each fractional
// component (LJ:128-135, AI:144-147).
__device__ __forceinline__ void mimg(double& dx, double& dy, double& dz, const double* hi, const double* h) {
    double s0 = dot3_rn(hi[0], hi[1], hi[2], dx, dy, dz);
    double s1 = dot3_rn(hi[3], hi[4], hi[5], dx, dy, dz);
    double s2 = dot3_rn(hi[6], hi[7], hi[8], dx, dy, dz);
    s0 = __dsub_rn(s0, round(s0));
    s1 = __dsub_rn(s1, round(s1));
    s2 = __dsub_rn(s2, round(s2));
    dx = dot3_rn(h[0], h[1], h[2], s0, s1, s2);
    dy = dot3_rn(h[3], h[4], h[5], s0, s1, s2);
    dz = dot3_rn(h[6], h[7], h[8], s0, s1, s2);
}

// LJ:114-117.
__device__ __forceinline__ double det9(const double* h) {
    double a = __dsub_rn(__dmul_rn(h[4], h[8]), __dmul_rn(h[5], h[7]));
    double b = __dsub_rn(__dmul_rn(h[3], h[8]), __dmul_rn(h[5], h[6]));
    double c = __dsub_rn(__dmul_rn(h[3], h[7]), __dmul_rn(h[4], h[6]));
    return __dadd_rn(__dsub_rn(__dmul_rn(h[0], a), __dmul_rn(h[1], b)), __dmul_rn(h[2], c));
}

__device__ __forceinline__ double cof_rn(double a, double b, double c, double d) {
    return __dsub_rn(__dmul_rn(a, b), __dmul_rn(c, d));
}

// LJ:120-124: adjugate times 1/det (IEEE division on the device).
__device__ __forceinline__ void inv9(const double* h, double* hi) {
    double id = __ddiv_rn(1.0, det9(h));
    hi[0] = __dmul_rn(id, cof_rn(h[4], h[8], h[5], h[7]));
    hi[1] = __dmul_rn(id, cof_rn(h[2], h[7], h[1], h[8]));
    hi[2] = __dmul_rn(id, cof_rn(h[1], h[5], h[2], h[4]));
    hi[3] = __dmul_rn(id, cof_rn(h[5], h[6], h[3], h[8]));
    hi[4] = __dmul_rn(id, cof_rn(h[0], h[8], h[2], h[6]));
    hi[5] = __dmul_rn(id, cof_rn(h[2], h[3], h[0], h[5]));
    hi[6] = __dmul_rn(id, cof_rn(h[3], h[7], h[4], h[6]));
    hi[7] = __dmul_rn(id, cof_rn(h[1], h[6], h[0], h[7]));
    hi[8] = __dmul_rn(id, cof_rn(h[0], h[4], h[1], h[3]));
}

// Fractional coordinates and the floor() wrap of apply_pbc (LJ:137-151).
__device__ __forceinline__ void wrap_point(double& x, double& y, double& z, const double* h, const double* hi) {
    double s0 = dot3_rn(hi[0], hi[1], hi[2], x, y, z);
    double s1 = dot3_rn(hi[3], hi[4], hi[5], x, y, z);
    double s2 = dot3_rn(hi[6], hi[7], hi[8], x, y, z);
    s0 = __dsub_rn(s0, floor(s0));
    s1 = __dsub_rn(s1, floor(s1));
    s2 = __dsub_rn(s2, floor(s2));
    x = dot3_rn(h[0], h[1], h[2], s0, s1, s2);
    y = dot3_rn(h[3], h[4], h[5], s0, s1, s2);
    z = dot3_rn(h[6], h[7], h[8], s0, s1, s2);
}

// ---- warp / block reductions with a fixed order (deterministic) ----------
template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Reduces NV values over the block and writes them to out[0..NV) from thread 0.
// Requires blockDim.x to be a multiple of 32 and <= 1024; `sm` holds
// 32*NV doubles.
template <int NV>
__device__ __forceinline__ void block_sum_store(double (&v)[NV], double* sm, double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) sm[warp * NV + k] = v[k];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double t = lane < nw ? sm[lane * NV + k] : 0.0;
            t = warp_sum(t);
            if (lane == 0) out[k] = t;
        }
    }
    __syncthreads();
}

}  // namespace fmd
