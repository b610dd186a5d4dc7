// rebo_fn.cuh -- REBO C-C pair functions and bond geometry shared by the
// plain REBO kernel (airebo.cu) and the learned bond-order path
// (surrogate.cu): parameters AI:110-116, cutoff and pair functions
// AI:164-191, bond vectors with the reference's min image (mimg9, AI:144-147).
#pragma once
#include <cmath>

#include "geom.cuh"
#include "kernels.h"

namespace fmd {
namespace rebo {

// REBO C-C parameters (AI:110-116).
constexpr double Q_CC = 0.3134602960833, A_CC = 10953.544162170, ALPHA_CC = 4.7465390606595;
constexpr double B1_CC = 12388.79197798, BETA1_CC = 4.7204523127;
constexpr double B2_CC = 17.56740646509, BETA2_CC = 1.4332132499;
constexpr double B3_CC = 30.71493208065, BETA3_CC = 1.3826912506;
constexpr double DMIN_CC = 1.7, DMAX_CC = 2.0, BO_DELTA = 0.5;
constexpr double G_A0 = 0.00020813, G_C0 = 330.0, G_D0 = 3.5;

__device__ __forceinline__ double sw_fc(double r) {
    if (r <= DMIN_CC) return 1.0;
    if (r >= DMAX_CC) return 0.0;
    return 0.5 * (1.0 + cos(kPi * (r - DMIN_CC) / (DMAX_CC - DMIN_CC)));
}
__device__ __forceinline__ double sw_dfc(double r) {
    if (r <= DMIN_CC || r >= DMAX_CC) return 0.0;
    return -0.5 * kPi / (DMAX_CC - DMIN_CC) * sin(kPi * (r - DMIN_CC) / (DMAX_CC - DMIN_CC));
}
__device__ __forceinline__ double ang_g(double x) {
    const double c2 = G_C0 * G_C0, d2 = G_D0 * G_D0, hh = 1.0 + x;
    return G_A0 * (1.0 + c2 / d2 - c2 / (d2 + hh * hh));
}
__device__ __forceinline__ double ang_dg(double x) {
    const double c2 = G_C0 * G_C0, d2 = G_D0 * G_D0, hh = 1.0 + x, dn = d2 + hh * hh;
    return G_A0 * 2.0 * c2 * hh / (dn * dn);
}
__device__ __forceinline__ double clamp1(double c) { return c < -1.0 ? -1.0 : (c > 1.0 ? 1.0 : c); }

__device__ __forceinline__ void load_cell(const double* __restrict__ hh, double* h, double* hi) {
#pragma unroll
    for (int k = 0; k < 9; k++) { h[k] = hh[k]; hi[k] = hh[9 + k]; }
}

__device__ __forceinline__ void bond_vec(const double* __restrict__ pos, int a, int b, const double* h,
                                         const double* hi, double& x, double& y, double& z) {
    x = __dsub_rn(pos[3 * b], pos[3 * a]);
    y = __dsub_rn(pos[3 * b + 1], pos[3 * a + 1]);
    z = __dsub_rn(pos[3 * b + 2], pos[3 * a + 2]);
    mimg(x, y, z, hi, h);
}

__device__ __forceinline__ void atomic_add3(double* F, int i, double x, double y, double z) {
    atomicAdd(&F[3 * i], x);
    atomicAdd(&F[3 * i + 1], y);
    atomicAdd(&F[3 * i + 2], z);
}

}  // namespace rebo
}  // namespace fmd
