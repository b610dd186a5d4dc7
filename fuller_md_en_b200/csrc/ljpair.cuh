// ljpair.cuh -- the shifted 12-6 LJ pair of the AIREBO and MM programs
// (AI:119-124, 441-446; MM:113-116) and the exact diagonal-cell minimum
// image, used by the list gathers (airebo.cu); the switched-LJ correction
// (rebo2.cu) takes the pair constants from here.
#pragma once
#include <cmath>
#include "geom.cuh"
#include "kernels.h"

namespace fmd {
namespace {

struct LJP {
    double sig2, c4, c24, rc2, vshift;
};

// Reference constants, computed with the reference's expressions.
__host__ __device__ inline LJP lj_params_dev(int ff) {
    LJP p;
    if (ff == FMD_FF_AIREBO) {  // AI:119-124
        const double sig = 3.40, eps = 2.84e-3, rc = 3.0 * sig;
        const double sr = sig / rc, sr2 = sr * sr, sr6 = sr2 * sr2 * sr2;
        p.sig2 = sig * sig; p.c4 = 4 * eps; p.c24 = 24 * eps; p.rc2 = rc * rc;
        p.vshift = 4 * eps * (sr6 * sr6 - sr6);
    } else {                    // MM:113-116
        const double sig = 3.431, eps = 2.635e-3, rc = 3.0 * sig;
        const double sr = 1.0 / 3.0, sr2 = sr * sr, sr6 = sr2 * sr2 * sr2;
        p.sig2 = sig * sig; p.c4 = 4 * eps; p.c24 = 24 * eps; p.rc2 = rc * rc;
        p.vshift = 4.0 * eps * (sr6 * sr6 - sr6);
    }
    return p;
}

// One component of the minimum image for a diagonal cell.  With zero
// off-diagonals the reference's s = hi0*dx + hi1*dy + hi2*dz and
// d = h0*s0 + h1*s1 + h2*s2 reduce exactly to these products (adding +-0
// changes nothing), so this is bitwise the reference's mimg.
// For |s| < 1.5 (always so for wrapped positions) round(s), half away from
// zero, is one of -1, 0, 1 and two comparisons give it exactly.
__device__ __forceinline__ double mimg1(double d, double hii, double hii_inv) {
    double s = __dmul_rn(hii_inv, d);
    double r = s >= 0.5 ? 1.0 : (s <= -0.5 ? -1.0 : 0.0);
    if (!(fabs(s) < 1.5)) r = round(s);
    s = __dsub_rn(s, r);
    return __dmul_rn(hii, s);
}

// The same image by one rounding instruction: rint (half to even) and the
// reference's round (half away from zero) differ only where s is a
// half-integer, and there both images lie half a cell edge away along this
// axis, so |d| and r^2 are the same under either and the pair is beyond the
// cutoff whenever half the narrowest edge exceeds it -- the only case this is
// used in.  Every other pair gets the identical image and d bit for bit.
__device__ __forceinline__ double mimg1_rint(double d, double hii, double hii_inv) {
    const double s = __dmul_rn(hii_inv, d);
    return __dmul_rn(hii, __dsub_rn(s, rint(s)));
}

// FP32 copies of the pair constants (FP32-pair precision).  sigma^2 is kept
// as a head + tail pair: its FP32 rounding would scale every s^6 by the same
// factor, a bias that the near-cancelling repulsive and attractive virial
// sums amplify about tenfold; c4 and c24 scale both parts alike and stay single.
struct LJF {
    float sig2, sig2_lo, c4, c24;
};

// One listed pair seen from atom i: d = r_j - r_i after the minimum image.
// The cutoff test is the reference's FP64 one in both precisions, so both
// modes interact through exactly the reference's pair set.  FP64: the
// reference's pair terms (AI:443-466) in the factored form below, equal to a
// few ulp.  FP32: the pair algebra (1/r^2, s^6, s^12, fm) in FP32; the
// minimum image, r^2, the force, energy and virial accumulation stay FP64.
// COUNT: this side counts energy and virial.
// FULL_VIRIAL (AIREBO's vir9, AI:455-466): the pair tensor d fm d^T is
// symmetric, so only its six distinct entries are accumulated, in acc[1],
// acc[2], acc[3], acc[5], acc[6], acc[9] (row-major W at acc[1..9]);
// lj_virial_mirror fills the lower triangle before the block sum.
template <bool FULL_VIRIAL, bool F32, bool COUNT>
__device__ __forceinline__ void lj_pair(double dx, double dy, double dz, const LJP& p, const LJF& pf,
                                        double& fx, double& fy, double& fz, double* acc) {
    double r2 = norm2_rn(dx, dy, dz);
    if (r2 > p.rc2) return;
    if (r2 < 0.25) r2 = 0.25;
    double fm, e = 0.0;
    if (F32) {
        const float ri2 = __frcp_rn((float)r2);
        const float s2 = fmaf(pf.sig2, ri2, pf.sig2_lo * ri2), s6 = s2 * s2 * s2, s12 = s6 * s6;
        fm = (double)(pf.c24 * (2.f * s12 - s6) * ri2);
        if (COUNT) e = (double)(pf.c4 * (s12 - s6)) - p.vshift;
    } else {
        // The reference's 24 eps (2 s^12 - s^6) / r^2 and 4 eps (s^12 - s^6)
        // (AI:443-445) as 24 eps s^6 (2 s^6 - 1) / r^2 and 4 eps s^6 (s^6 - 1),
        // with s^2 = sigma^2 / r^2 formed from the reciprocal approximation y
        // and its refinement c directly (sigma^2 y (1 + c)): the same values
        // to a few ulp, by a dependency chain four operations shorter.
        // 1/r^2 = y (1 + c), c = e + e^2, e = 1 - r^2 y: one third-order step
        // (the series of 1/(1 - e) to second order) cubes the approximation's
        // error, 2.2e-16 relative at most over r^2 in [0.25, 110] (measured on
        // B200), in place of a full IEEE division.
        double y;
        asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(r2));
        const double e0 = fma(-r2, y, 1.0), c = fma(e0, e0, e0);
        const double ri2 = fma(y, c, y), sy = p.sig2 * y;
        const double s2 = fma(sy, c, sy), s6 = s2 * s2 * s2;
        fm = (p.c24 * ri2 * s6) * fma(2.0, s6, -1.0);
        if (COUNT) e = p.c4 * s6 * (s6 - 1.0) - p.vshift;
    }
    if (COUNT && FULL_VIRIAL) {
        const double gx = fm * dx, gy = fm * dy, gz = fm * dz;
        fx -= gx; fy -= gy; fz -= gz;
        acc[0] += e;
        acc[1] += dx * gx; acc[2] += dx * gy; acc[3] += dx * gz;
        acc[5] += dy * gy; acc[6] += dy * gz;
        acc[9] += dz * gz;
        return;
    }
    fx -= fm * dx; fy -= fm * dy; fz -= fm * dz;
    if (COUNT) {
        acc[0] += e;
        acc[1] += dx * fm * dx;
        acc[5] += dy * fm * dy;
        acc[9] += dz * fm * dz;
    }
}

// Lower triangle of the symmetric virial accumulated by lj_pair<true, ...>.
template <bool FULL_VIRIAL>
__device__ __forceinline__ void lj_virial_mirror(double* acc) {
    if (FULL_VIRIAL) { acc[4] = acc[2]; acc[7] = acc[3]; acc[8] = acc[6]; }
}

}  // namespace
}  // namespace fmd
