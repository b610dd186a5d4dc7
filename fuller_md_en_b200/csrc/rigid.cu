// rigid.cu -- rigid-body site-site LJ (LJ:271-400, CORE:346-444).
//
// One CTA per molecule i.  Its lab-frame sites R(q_i) b_a are computed once
// into shared memory; each listed neighbour j whose COM image lies within
// rmcut has its sites staged in shared memory too (two neighbours in flight
// per CTA: threads [0,TS) and [TS,2TS) each own one neighbour slot).  Thread a
// of a slot owns site a of molecule i and loops over the 60 sites b of j,
// reading them as shared-memory broadcasts.  Force, torque, virial and
// energy are accumulated per thread in FP64 and reduced over the CTA in a
// fixed order (deterministic, no atomics: the list is symmetric, so every
// molecule owns its own sums exactly as in the reference).
//
// Precision:
//   FMD_PREC_FP64       site offsets, pair distance, cutoff and LJ in FP64 with
//                       the reference's operation order for every decision;
//   FMD_PREC_FP32_PAIR  COM image and cutoff skip in FP64, site offsets and
//                       pair arithmetic in FP32, per-neighbour FP32 sums folded
//                       into FP64 per-molecule accumulators.
#include <cmath>
#include "kernels.h"
#include "geom.cuh"

namespace fmd {
namespace {

constexpr double kSig = 3.431, kEps = 2.635e-3;   // LJ:103

struct RigidConst {
    double sig2, rcut2, c24, c4, vshift;
};

RigidConst rigid_const() {
    RigidConst c;
    const double rcut = 3.0 * kSig;
    const double sr = 1.0 / 3.0, sr2 = sr * sr, sr6 = sr2 * sr2 * sr2;
    c.sig2 = kSig * kSig;
    c.rcut2 = rcut * rcut;
    c.c24 = 24.0 * kEps;
    c.c4 = 4.0 * kEps;
    c.vshift = 4.0 * kEps * (sr6 * sr6 - sr6);
    return c;
}

// R(q) (LJ:155-159) with reference rounding.
__device__ __forceinline__ void quat_rot(const double* q, double* R) {
    const double w = q[0], x = q[1], y = q[2], z = q[3];
    R[0] = __dsub_rn(1.0, __dmul_rn(2.0, __dadd_rn(__dmul_rn(y, y), __dmul_rn(z, z))));
    R[1] = __dmul_rn(2.0, __dsub_rn(__dmul_rn(x, y), __dmul_rn(w, z)));
    R[2] = __dmul_rn(2.0, __dadd_rn(__dmul_rn(x, z), __dmul_rn(w, y)));
    R[3] = __dmul_rn(2.0, __dadd_rn(__dmul_rn(x, y), __dmul_rn(w, z)));
    R[4] = __dsub_rn(1.0, __dmul_rn(2.0, __dadd_rn(__dmul_rn(x, x), __dmul_rn(z, z))));
    R[5] = __dmul_rn(2.0, __dsub_rn(__dmul_rn(y, z), __dmul_rn(w, x)));
    R[6] = __dmul_rn(2.0, __dsub_rn(__dmul_rn(x, z), __dmul_rn(w, y)));
    R[7] = __dmul_rn(2.0, __dadd_rn(__dmul_rn(y, z), __dmul_rn(w, x)));
    R[8] = __dsub_rn(1.0, __dmul_rn(2.0, __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y))));
}

template <class P> struct Site;
template <> struct Site<double> { double x, y, z, pad; };
template <> struct __align__(16) Site<float> { float x, y, z, pad; };

constexpr int kMaxSites = 96;   // up to C84 (natom <= 84), padded to warps

template <class P>
__global__ void __launch_bounds__(2 * kMaxSites)
k_rigid(const double* __restrict__ pos, const double* __restrict__ qv, const double* __restrict__ body,
        const double* __restrict__ hh, const int* __restrict__ cnt, const int* __restrict__ list, int cap,
        int n, int natom, int ts, double rmcut2, RigidConst rc, double* __restrict__ F,
        double* __restrict__ T, double* __restrict__ part) {
    __shared__ Site<P> lab_i[kMaxSites];
    __shared__ Site<P> lab_j[2][kMaxSites];
    __shared__ double sm[32 * 16];
    const int i = blockIdx.x;
    const int slot = threadIdx.x / ts, a = threadIdx.x % ts;
    double h[9], hi[9];
#pragma unroll
    for (int k = 0; k < 9; k++) { h[k] = hh[k]; hi[k] = hh[9 + k]; }

    double R[9];
    quat_rot(qv + 4 * i, R);
    if (slot == 0 && a < natom) {
        const double bx = body[3 * a], by = body[3 * a + 1], bz = body[3 * a + 2];
        Site<P> s;
        s.x = (P)dot3_rn(R[0], R[1], R[2], bx, by, bz);
        s.y = (P)dot3_rn(R[3], R[4], R[5], bx, by, bz);
        s.z = (P)dot3_rn(R[6], R[7], R[8], bx, by, bz);
        s.pad = 0;
        lab_i[a] = s;
    }
    const double pix = pos[3 * i], piy = pos[3 * i + 1], piz = pos[3 * i + 2];
    double acc[16];   // F(3) T(3) W(9) E
#pragma unroll
    for (int k = 0; k < 16; k++) acc[k] = 0.0;
    const int nn = cnt[i];
    __syncthreads();
    const Site<P> ra = lab_i[a < natom ? a : 0];

    for (int k0 = 0; k0 < nn; k0 += 2) {
        const int k = k0 + slot;
        bool valid = k < nn;
        double mx = 0, my = 0, mz = 0;
        if (valid) {
            const int j = list[(size_t)i * cap + k];
            mx = __dsub_rn(pos[3 * j], pix);
            my = __dsub_rn(pos[3 * j + 1], piy);
            mz = __dsub_rn(pos[3 * j + 2], piz);
            mimg(mx, my, mz, hi, h);
            valid = !(norm2_rn(mx, my, mz) > rmcut2);
            if (valid && a < natom) {
                double Rj[9];
                quat_rot(qv + 4 * j, Rj);
                const double bx = body[3 * a], by = body[3 * a + 1], bz = body[3 * a + 2];
                Site<P> s;
                s.x = (P)dot3_rn(Rj[0], Rj[1], Rj[2], bx, by, bz);
                s.y = (P)dot3_rn(Rj[3], Rj[4], Rj[5], bx, by, bz);
                s.z = (P)dot3_rn(Rj[6], Rj[7], Rj[8], bx, by, bz);
                s.pad = 0;
                lab_j[slot][a] = s;
            }
        }
        __syncthreads();
        if (valid && a < natom) {
            const Site<P>* sj = lab_j[slot];
            if constexpr (sizeof(P) == 8) {
                // FP64: reference order ((dm + r_b) - r_a) for every decision.
                double f0 = 0, f1 = 0, f2 = 0, w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, e = 0;
                const double rax = (double)ra.x, ray = (double)ra.y, raz = (double)ra.z;
                for (int b = 0; b < natom; b++) {
                    const Site<P> rb = sj[b];
                    const double dx = __dsub_rn(__dadd_rn(mx, (double)rb.x), rax);
                    const double dy = __dsub_rn(__dadd_rn(my, (double)rb.y), ray);
                    const double dz = __dsub_rn(__dadd_rn(mz, (double)rb.z), raz);
                    double r2 = norm2_rn(dx, dy, dz);
                    if (r2 < rc.rcut2) {
                        if (r2 < 0.25) r2 = 0.25;
                        const double ri2 = 1.0 / r2, s2 = rc.sig2 * ri2, s6 = s2 * s2 * s2, s12 = s6 * s6;
                        const double fm = rc.c24 * (2.0 * s12 - s6) * ri2;
                        const double fx = fm * dx, fy = fm * dy, fz = fm * dz;
                        f0 -= fx; f1 -= fy; f2 -= fz;
                        e += 0.5 * (rc.c4 * (s12 - s6) - rc.vshift);
                        w[0] += 0.5 * dx * fx; w[1] += 0.5 * dx * fy; w[2] += 0.5 * dx * fz;
                        w[3] += 0.5 * dy * fx; w[4] += 0.5 * dy * fy; w[5] += 0.5 * dy * fz;
                        w[6] += 0.5 * dz * fx; w[7] += 0.5 * dz * fy; w[8] += 0.5 * dz * fz;
                    }
                }
                acc[0] += f0; acc[1] += f1; acc[2] += f2;
                // torque -= r_a x f, summed over b: r_a x (sum f) with f = -F contribution
                acc[3] += ray * f2 - raz * f1;
                acc[4] += raz * f0 - rax * f2;
                acc[5] += rax * f1 - ray * f0;
#pragma unroll
                for (int q = 0; q < 9; q++) acc[6 + q] += w[q];
                acc[15] += e;
            } else {
                // The COM image (up to ~18 A) rounded to FP32 would carry a
                // 1e-6 A error shared by all 3600 site pairs of the molecule
                // pair; split it into hi + lo parts and add the small site
                // difference first so each pair distance keeps ~1e-7 relative
                // accuracy.
                const float mxh = (float)mx, myh = (float)my, mzh = (float)mz;
                const float mxl = (float)(mx - (double)mxh), myl = (float)(my - (double)myh),
                            mzl = (float)(mz - (double)mzh);
                const float rax = (float)ra.x, ray = (float)ra.y, raz = (float)ra.z;
                const float sig2 = (float)rc.sig2, rcut2 = (float)rc.rcut2, c24 = (float)rc.c24,
                            c4 = (float)rc.c4, vsh = (float)rc.vshift;
                float f0 = 0, f1 = 0, f2 = 0;
                for (int b = 0; b < natom; b++) {
                    const Site<P> rb = sj[b];
                    const float dx = (mxh + ((float)rb.x - rax)) + mxl;
                    const float dy = (myh + ((float)rb.y - ray)) + myl;
                    const float dz = (mzh + ((float)rb.z - raz)) + mzl;
                    float r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 < rcut2) {
                        r2 = fmaxf(r2, 0.25f);
                        const float ri2 = 1.0f / r2, s2 = sig2 * ri2, s6 = s2 * s2 * s2, s12 = s6 * s6;
                        const float fm = c24 * (2.0f * s12 - s6) * ri2;
                        const float fx = fm * dx, fy = fm * dy, fz = fm * dz;
                        f0 -= fx; f1 -= fy; f2 -= fz;
                        // energy and virial: FP32 pair terms, FP64 sums, halved
                        // for the symmetric list (LJ:339-341)
                        const float hx = 0.5f * dx, hy = 0.5f * dy, hz = 0.5f * dz;
                        acc[15] += (double)(0.5f * (c4 * (s12 - s6) - vsh));
                        acc[6] += (double)(hx * fx); acc[7] += (double)(hx * fy); acc[8] += (double)(hx * fz);
                        acc[9] += (double)(hy * fx); acc[10] += (double)(hy * fy); acc[11] += (double)(hy * fz);
                        acc[12] += (double)(hz * fx); acc[13] += (double)(hz * fy); acc[14] += (double)(hz * fz);
                    }
                }
                const double rad[3] = {(double)ra.x, (double)ra.y, (double)ra.z};
                acc[0] += f0; acc[1] += f1; acc[2] += f2;
                acc[3] += rad[1] * (double)f2 - rad[2] * (double)f1;
                acc[4] += rad[2] * (double)f0 - rad[0] * (double)f2;
                acc[5] += rad[0] * (double)f1 - rad[1] * (double)f0;
            }
        }
        __syncthreads();
    }
    double tot[16];
    block_sum_store<16>(acc, sm, tot);
    if (threadIdx.x == 0) {
        F[3 * i] = tot[0]; F[3 * i + 1] = tot[1]; F[3 * i + 2] = tot[2];
        T[3 * i] = tot[3]; T[3 * i + 1] = tot[4]; T[3 * i + 2] = tot[5];
        double* o = part + (size_t)i * kNV;
        o[0] = tot[15];
#pragma unroll
        for (int q = 0; q < 9; q++) o[1 + q] = tot[6 + q];
    }
}

}  // namespace

int rigid_grid(int n) { return n; }

cudaError_t rigid_launch(int precision, const double* pos, const double* qv, const double* body,
                         const double* hh, const int* cnt, const int* list, int cap, int n, int natom,
                         double rmcut2, double* F, double* T, double* part, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (natom < 1 || natom > kMaxSites) return cudaErrorInvalidValue;
    const int ts = ((natom + 31) / 32) * 32;
    const RigidConst rc = rigid_const();
    if (precision == FMD_PREC_FP32_PAIR)
        k_rigid<float><<<n, 2 * ts, 0, st>>>(pos, qv, body, hh, cnt, list, cap, n, natom, ts, rmcut2, rc, F, T, part);
    else
        k_rigid<double><<<n, 2 * ts, 0, st>>>(pos, qv, body, hh, cnt, list, cap, n, natom, ts, rmcut2, rc, F, T, part);
    return cudaGetLastError();
}

}  // namespace fmd
