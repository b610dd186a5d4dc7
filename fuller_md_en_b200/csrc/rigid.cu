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
#include <algorithm>
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
constexpr int kRigidMaxNeigh = 128;   // list width the warp kernel accepts (the reference's is 80)

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

// ---------------------------------------------------------------------------
// Warp-per-neighbour variant.  k_rigid_lab writes every molecule's lab-frame
// sites once per step (the reference computes the whole lab frame first too,
// LJ:276-291).  In k_rigid_w one CTA owns molecule i; each warp takes one
// listed neighbour j at a time, copies j's sites from the lab array into its
// own shared-memory slice with coalesced 16/32-byte loads, and lane l handles
// sites l and l + 32 of i against all sites of j -- no block-wide barrier in
// the neighbour loop.  Per-neighbour partial sums stay in the pair precision
// and are folded into FP64 per-molecule accumulators; the CTA reduces them
// in a fixed order.
template <class P>
__global__ void __launch_bounds__(256)
k_rigid_lab(const double* __restrict__ qv, const double* __restrict__ body, int n, int natom,
            Site<P>* __restrict__ lab) {
    const long long tot = (long long)n * natom;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / natom), a = (int)(t % natom);
        double R[9];
        quat_rot(qv + 4 * i, R);
        const double bx = body[3 * a], by = body[3 * a + 1], bz = body[3 * a + 2];
        Site<P> s;
        s.x = (P)dot3_rn(R[0], R[1], R[2], bx, by, bz);
        s.y = (P)dot3_rn(R[3], R[4], R[5], bx, by, bz);
        s.z = (P)dot3_rn(R[6], R[7], R[8], bx, by, bz);
        s.pad = 0;
        lab[t] = s;
    }
}

// W warps per molecule; MINB resident blocks per SM requested from the
// compiler (a register cap: 0 leaves the register count free).
template <class P, int W, int MINB>
__global__ void __launch_bounds__(32 * W, MINB)
k_rigid_w(const double* __restrict__ pos, const Site<P>* __restrict__ lab, const double* __restrict__ hh,
          const int* __restrict__ cnt, const int* __restrict__ list, int cap, int n, int natom, double rmcut2,
          RigidConst rc, double* __restrict__ F, double* __restrict__ T, double* __restrict__ part) {
    constexpr int kRigidWarps = W;
    __shared__ Site<P> lab_i[2 * 32];
    __shared__ Site<P> lab_j[kRigidWarps][2 * 32];
    __shared__ double sm[32 * 16];
    __shared__ double s_hh[18];
    __shared__ float s_cost[kRigidMaxNeigh];
    __shared__ int s_order[kRigidMaxNeigh];
    const int i = blockIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x < 18) s_hh[threadIdx.x] = hh[threadIdx.x];
    for (int a = threadIdx.x; a < natom; a += blockDim.x) lab_i[a] = lab[(size_t)i * natom + a];
    __syncthreads();
    const double* h = s_hh;
    const double* hi = s_hh + 9;
    const double pix = pos[3 * i], piy = pos[3 * i + 1], piz = pos[3 * i + 2];
    const int a0 = lane, a1 = lane + 32;
    const bool v0 = a0 < natom, v1 = a1 < natom;
    const Site<P> r0 = lab_i[v0 ? a0 : 0], r1 = lab_i[v1 ? a1 : 0];
    // Site screen: a pair within the cutoff has |m + r_b| <= |d| + |r_a| <
    // rcut + R, with m the COM image, d the pair vector and R the largest site
    // radius (all molecules share one body, so i's own sites give it).  Only
    // j's sites within rcut + R (+ a margin far above the rounding of either
    // precision) of i's centre enter the pair loop, in ascending order, so
    // the pairs that count and the order of their sums are unchanged.
    double rmax2 = 0.0;
    {
        const double q0 = v0 ? (double)r0.x * r0.x + (double)r0.y * r0.y + (double)r0.z * r0.z : 0.0;
        const double q1 = v1 ? (double)r1.x * r1.x + (double)r1.y * r1.y + (double)r1.z * r1.z : 0.0;
        rmax2 = fmax(q0, q1);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) rmax2 = fmax(rmax2, __shfl_xor_sync(kFull, rmax2, o));
    }
    const double screen = sqrt(rc.rcut2) + sqrt(rmax2) + 1e-2, screen2 = screen * screen;
    const unsigned lt = (1u << lane) - 1u;
    // Neighbour order: a neighbour's cost is about the number of its sites
    // inside the screen radius -- the fraction of a sphere of radius R at
    // distance d inside a sphere of radius S about i's centre, (S^2 - (d -
    // R)^2) / (4 d R) -- plus its staging.  Ranked by cost (ties by list
    // position) and dealt to the warps in snake order, the same assignment
    // on every run, so the summation order stays fixed.
    const int nn = cnt[i];
    if (nn > kRigidMaxNeigh) return;                  // the lists are built with cap <= kRigidMaxNeigh
    {
        const double R = sqrt(rmax2);
        for (int k = threadIdx.x; k < nn; k += blockDim.x) {
            const int j = list[(size_t)i * cap + k];
            double mx = __dsub_rn(pos[3 * j], pix), my = __dsub_rn(pos[3 * j + 1], piy),
                   mz = __dsub_rn(pos[3 * j + 2], piz);
            mimg(mx, my, mz, hi, h);
            const double d2 = norm2_rn(mx, my, mz);
            float cost = 0.f;
            if (!(d2 > rmcut2)) {
                const double d = sqrt(d2);
                const double f = d + R <= screen ? 1.0 : (d - R >= screen ? 0.0
                                 : (screen2 - (d - R) * (d - R)) / (4.0 * d * R));
                cost = 8.f + (float)(natom * fmin(1.0, fmax(0.0, f)));
            }
            s_cost[k] = cost;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < nn; k += blockDim.x) {
            const float ck = s_cost[k];
            int rank = 0;
            for (int u = 0; u < nn; u++) {
                const float cu = s_cost[u];
                rank += cu > ck || (cu == ck && u < k);
            }
            s_order[rank] = k;
        }
        __syncthreads();
    }
    double acc[16];   // F(3) T(3) W(9) E
#pragma unroll
    for (int k = 0; k < 16; k++) acc[k] = 0.0;
    const float sig2 = (float)rc.sig2, sig2_lo = (float)(rc.sig2 - (double)(float)rc.sig2);
    const float rcut2f = (float)rc.rcut2, c24f = (float)rc.c24, c4f = (float)rc.c4;
    Site<P>* sj = lab_j[w];
    for (int p0 = 0; p0 < nn; p0 += kRigidWarps) {
        // snake: warp w takes position p0 + w on even rounds, p0 + W-1-w on odd ones
        const int p = p0 + (((p0 / kRigidWarps) & 1) ? kRigidWarps - 1 - w : w);
        if (p >= nn) continue;
        const int j = list[(size_t)i * cap + s_order[p]];
        double mx = __dsub_rn(pos[3 * j], pix), my = __dsub_rn(pos[3 * j + 1], piy), mz = __dsub_rn(pos[3 * j + 2], piz);
        mimg(mx, my, mz, hi, h);
        if (norm2_rn(mx, my, mz) > rmcut2) continue;             // warp-uniform (LJ:320)
        __syncwarp();
        // j's sites a0, a1 of this lane, kept by the screen, stored compacted
        int nb;
        {
            Site<P> q[2];
            bool keep[2];
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int b = s ? a1 : a0;
                keep[s] = s ? v1 : v0;
                if (!keep[s]) continue;
                q[s] = lab[(size_t)j * natom + b];
                const double ux = (double)q[s].x + mx, uy = (double)q[s].y + my, uz = (double)q[s].z + mz;
                keep[s] = ux * ux + uy * uy + uz * uz < screen2;
                if constexpr (sizeof(P) == 4) {
                    // FP32 pairs: j's sites moved by the COM image m in FP64 and
                    // rounded once, so each pair distance is one subtraction; the
                    // rounding error is independent per site.
                    q[s].x = (float)ux; q[s].y = (float)uy; q[s].z = (float)uz; q[s].pad = 0.f;
                }
            }
            const unsigned m0 = __ballot_sync(kFull, keep[0]), m1 = __ballot_sync(kFull, keep[1]);
            if (keep[0]) sj[__popc(m0 & lt)] = q[0];
            if (keep[1]) sj[__popc(m0) + __popc(m1 & lt)] = q[1];
            nb = __popc(m0) + __popc(m1);
        }
        __syncwarp();
        if (nb == 0) continue;                                   // warp-uniform
        // per-neighbour partial sums for sites a0 and a1
        P f[2][3] = {{0, 0, 0}, {0, 0, 0}}, wv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, e = 0;
        if constexpr (sizeof(P) == 8) {
            for (int b = 0; b < nb; b++) {
                const Site<P> rb = sj[b];
#pragma unroll
                for (int s = 0; s < 2; s++) {
                    const Site<P>& ra = s ? r1 : r0;
                    if (!(s ? v1 : v0)) continue;
                    // FP64: reference order ((dm + r_b) - r_a) for every decision (LJ:330-336)
                    const double dx = __dsub_rn(__dadd_rn(mx, rb.x), ra.x);
                    const double dy = __dsub_rn(__dadd_rn(my, rb.y), ra.y);
                    const double dz = __dsub_rn(__dadd_rn(mz, rb.z), ra.z);
                    double r2 = norm2_rn(dx, dy, dz);
                    if (r2 < rc.rcut2) {
                        if (r2 < 0.25) r2 = 0.25;
                        const double ri2 = 1.0 / r2, s2 = rc.sig2 * ri2, s6 = s2 * s2 * s2, s12 = s6 * s6;
                        const double fm = rc.c24 * (2.0 * s12 - s6) * ri2;
                        const double fx = fm * dx, fy = fm * dy, fz = fm * dz;
                        f[s][0] -= fx; f[s][1] -= fy; f[s][2] -= fz;
                        e += 0.5 * (rc.c4 * (s12 - s6) - rc.vshift);
                        wv[0] += 0.5 * dx * fx; wv[1] += 0.5 * dx * fy; wv[2] += 0.5 * dx * fz;
                        wv[3] += 0.5 * dy * fx; wv[4] += 0.5 * dy * fy; wv[5] += 0.5 * dy * fz;
                        wv[6] += 0.5 * dz * fx; wv[7] += 0.5 * dz * fy; wv[8] += 0.5 * dz * fz;
                    }
                }
            }
        } else {
            float eterm = 0.f;
            float wxx = 0.f, wyy = 0.f, wzz = 0.f, wxy = 0.f, wxz = 0.f, wyz = 0.f;
            int npair = 0;
            for (int b = 0; b < nb; b++) {
                const Site<P> rb = sj[b];
#pragma unroll
                for (int s = 0; s < 2; s++) {
                    const Site<P>& ra = s ? r1 : r0;
                    if (!(s ? v1 : v0)) continue;
                    const float dx = rb.x - ra.x, dy = rb.y - ra.y, dz = rb.z - ra.z;
                    float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                    if (r2 < rcut2f) {
                        r2 = fmaxf(r2, 0.25f);
                        const float ri2 = 1.0f / r2, s2 = fmaf(sig2, ri2, sig2_lo * ri2), s6 = s2 * s2 * s2,
                                    s12 = s6 * s6;
                        const float fm = c24f * fmaf(2.0f, s12, -s6) * ri2;
                        const float fx = fm * dx, fy = fm * dy, fz = fm * dz;
                        f[s][0] -= fx; f[s][1] -= fy; f[s][2] -= fz;
                        eterm = fmaf(c4f, s12 - s6, eterm);
                        npair++;
                        // fm d (x) d is symmetric: six components
                        wxx = fmaf(dx, fx, wxx); wyy = fmaf(dy, fy, wyy); wzz = fmaf(dz, fz, wzz);
                        wxy = fmaf(dx, fy, wxy); wxz = fmaf(dx, fz, wxz); wyz = fmaf(dy, fz, wyz);
                    }
                }
            }
            wv[0] = wxx; wv[4] = wyy; wv[8] = wzz;
            wv[1] = wv[3] = wxy; wv[2] = wv[6] = wxz; wv[5] = wv[7] = wyz;
            // energy and virial halved for the symmetric list (LJ:339-341); the
            // shift in FP64 once per neighbour
            e = 0.5f * eterm;
            acc[15] -= 0.5 * rc.vshift * npair;
#pragma unroll
            for (int q = 0; q < 9; q++) wv[q] *= 0.5f;
        }
#pragma unroll
        for (int s = 0; s < 2; s++) {
            if (!(s ? v1 : v0)) continue;
            const Site<P>& ra = s ? r1 : r0;
            const double fx = (double)f[s][0], fy = (double)f[s][1], fz = (double)f[s][2];
            const double rx = (double)ra.x, ry = (double)ra.y, rz = (double)ra.z;
            acc[0] += fx; acc[1] += fy; acc[2] += fz;
            // torque -= r_a x f with f the force on i's site (LJ:337)
            acc[3] += ry * fz - rz * fy;
            acc[4] += rz * fx - rx * fz;
            acc[5] += rx * fy - ry * fx;
        }
#pragma unroll
        for (int q = 0; q < 9; q++) acc[6 + q] += (double)wv[q];
        acc[15] += (double)e;
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

// Site pairs within the cutoff, each molecule pair once (j > i), by the
// reference's FP64 test on the lab-frame sites (LJ:320-336): the algorithmic
// work count of the site-pair kernel (72 FLOP per counted pair).  One CTA
// per molecule, one warp per listed neighbour.
__global__ void __launch_bounds__(128)
k_rigid_count(const double* __restrict__ pos, const Site<double>* __restrict__ lab, const double* __restrict__ hh,
              const int* __restrict__ cnt, const int* __restrict__ list, int cap, int natom, double rmcut2,
              double rcut2, unsigned long long* __restrict__ total) {
    const int i = blockIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, W = blockDim.x >> 5;
    const double* h = hh;
    const double* hi = hh + 9;
    const double pix = pos[3 * i], piy = pos[3 * i + 1], piz = pos[3 * i + 2];
    unsigned long long c = 0;
    for (int k = w; k < cnt[i]; k += W) {
        const int j = list[(size_t)i * cap + k];
        if (j <= i) continue;
        double mx = __dsub_rn(pos[3 * j], pix), my = __dsub_rn(pos[3 * j + 1], piy), mz = __dsub_rn(pos[3 * j + 2], piz);
        mimg(mx, my, mz, hi, h);
        if (norm2_rn(mx, my, mz) > rmcut2) continue;
        for (int a = 0; a < natom; a++) {
            const Site<double> ra = lab[(size_t)i * natom + a];
            for (int b = lane; b < natom; b += 32) {
                const Site<double> rb = lab[(size_t)j * natom + b];
                const double dx = __dsub_rn(__dadd_rn(mx, rb.x), ra.x);
                const double dy = __dsub_rn(__dadd_rn(my, rb.y), ra.y);
                const double dz = __dsub_rn(__dadd_rn(mz, rb.z), ra.z);
                c += norm2_rn(dx, dy, dz) < rcut2;
            }
        }
    }
    c = __reduce_add_sync(kFull, (unsigned)c);
    if (lane == 0 && c) atomicAdd(total, c);
}

}  // namespace

int rigid_grid(int n) { return n; }

cudaError_t rigid_count_pairs(const double* pos, const double* qv, const double* body, const double* hh,
                              const int* cnt, const int* list, int cap, int n, int natom, double rmcut2, double* lab,
                              unsigned long long* total, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (natom < 1 || natom > kMaxSites || !lab) return cudaErrorInvalidValue;
    const RigidConst rc = rigid_const();
    const int lb = (int)std::min<long long>(((long long)n * natom + 255) / 256, kSMs * 16);
    Site<double>* sl = reinterpret_cast<Site<double>*>(lab);
    k_rigid_lab<double><<<lb, 256, 0, st>>>(qv, body, n, natom, sl);
    cudaMemsetAsync(total, 0, sizeof(unsigned long long), st);
    k_rigid_count<<<n, 128, 0, st>>>(pos, sl, hh, cnt, list, cap, natom, rmcut2, rc.rcut2, total);
    return cudaGetLastError();
}

cudaError_t rigid_launch(int precision, const double* pos, const double* qv, const double* body,
                         const double* hh, const int* cnt, const int* list, int cap, int n, int natom,
                         double rmcut2, double* F, double* T, double* part, cudaStream_t st, double* lab,
                         int shape) {
    if (n <= 0) return cudaSuccess;
    if (natom < 1 || natom > kMaxSites) return cudaErrorInvalidValue;
    const RigidConst rc = rigid_const();
    if (lab != nullptr && natom <= 64 && cap <= kRigidMaxNeigh) {
        const int lb = (int)std::min<long long>(((long long)n * natom + 255) / 256, kSMs * 16);
#define FMD_RW(P, W, MB) \
    k_rigid_w<P, W, MB><<<n, 32 * W, 0, st>>>(pos, reinterpret_cast<const Site<P>*>(lab), hh, cnt, list, cap, n, natom, \
                                              rmcut2, rc, F, T, part)
        if (precision == FMD_PREC_FP32_PAIR) {
            k_rigid_lab<float><<<lb, 256, 0, st>>>(qv, body, n, natom, reinterpret_cast<Site<float>*>(lab));
            if (shape == 1) FMD_RW(float, 4, 4); else if (shape == 2) FMD_RW(float, 8, 2); else FMD_RW(float, 4, 1);
        } else {
            k_rigid_lab<double><<<lb, 256, 0, st>>>(qv, body, n, natom, reinterpret_cast<Site<double>*>(lab));
            if (shape == 1) FMD_RW(double, 4, 4); else if (shape == 2) FMD_RW(double, 8, 2); else FMD_RW(double, 4, 1);
        }
#undef FMD_RW
        return cudaGetLastError();
    }
    const int ts = ((natom + 31) / 32) * 32;
    if (precision == FMD_PREC_FP32_PAIR)
        k_rigid<float><<<n, 2 * ts, 0, st>>>(pos, qv, body, hh, cnt, list, cap, n, natom, ts, rmcut2, rc, F, T, part);
    else
        k_rigid<double><<<n, 2 * ts, 0, st>>>(pos, qv, body, hh, cnt, list, cap, n, natom, ts, rmcut2, rc, F, T, part);
    return cudaGetLastError();
}

}  // namespace fmd
