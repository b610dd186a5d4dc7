// airebo.cu -- the simplified AIREBO force field (AI:275-495) and the
// half-list shifted LJ shared with the MM program (MM:711-764).
//
// REBO (a7): one thread per atom i walks its bonds j>i (3 per atom in a
// fullerene).  The bond order needs both ends' neighbourhoods, and the
// reference's three-body forces land on the neighbours k of i and l of j, so
// forces are scattered with FP64 atomics; energy and virial go to per-block
// partials that a fixed-order reduction sums.
//
// LJ (a8/a14): a deterministic gather.  The reference visits each listed pair
// once and scatters F_j with atomics; here each atom's warp visits its own
// outgoing entries (the reference row, j>i) and its incoming entries (the
// transposed rows, j<i), accumulates only its own force, and counts energy and
// virial on the outgoing side only, so every listed pair contributes exactly
// once, as in the reference.  The cutoff decision uses the reference's
// operation order, and mimg(-d) == -mimg(d) bitwise, so both sides of a pair
// always agree on whether it interacts.
#include <cmath>
#include "kernels.h"
#include "geom.cuh"
#include "rebo_fn.cuh"

namespace fmd {
namespace {

using namespace rebo;

// Sum over the centre's other neighbours of fc * G(cos theta) (AI:301-309).
__device__ double bo_sum(const double* __restrict__ pos, const int* __restrict__ cnt,
                         const int* __restrict__ list, int cap, const double* h, const double* hi,
                         int c, int skip, double bx, double by, double bz, double rb) {
    double gs = 0.0;
    const int m = cnt[c];
    for (int kn = 0; kn < m; kn++) {
        const int k = list[(size_t)c * cap + kn];
        if (k == skip) continue;
        double kx, ky, kz;
        bond_vec(pos, c, k, h, hi, kx, ky, kz);
        const double rk = sqrt(norm2_rn(kx, ky, kz));
        if (rk > DMAX_CC) continue;
        const double fk = sw_fc(rk);
        if (fk < 1e-15) continue;
        const double ct = clamp1((bx * kx + by * ky + bz * kz) / (rb * rk));
        gs += fk * ang_g(ct);
    }
    return gs;
}

// Reference three-body forces on the neighbours of centre c (AI:361-419).
// b = (1+gs)^-1/2 is passed in, so db/dgs = -1/2 (1+gs)^-3/2 = -b / (2 (1+gs)).
__device__ __forceinline__ void bo_three_body(double* __restrict__ F, const double* __restrict__ pos,
                              const int* __restrict__ cnt, const int* __restrict__ list, int cap,
                              const double* h, const double* hi, int c, int skip, double bx, double by,
                              double bz, double rb, double ux, double uy, double uz, double gs, double b,
                              double fcut, double va) {
    if (!(fabs(gs) > 1e-20 && va > 1e-20)) return;
    const double dbp = -BO_DELTA * b / (1.0 + gs);
    const double vh = 0.5 * fcut * va;
    const double coeff = -vh * dbp;
    const int m = cnt[c];
    double fcx = 0.0, fcy = 0.0, fcz = 0.0;
    for (int kn = 0; kn < m; kn++) {
        const int k = list[(size_t)c * cap + kn];
        if (k == skip) continue;
        double kx, ky, kz;
        bond_vec(pos, c, k, h, hi, kx, ky, kz);
        const double rk = sqrt(norm2_rn(kx, ky, kz));
        if (rk > DMAX_CC) continue;
        const double fck = sw_fc(rk);
        if (fck < 1e-15) continue;
        const double dfck = sw_dfc(rk);
        const double rki = 1.0 / rk;
        const double rx = kx * rki, ry = ky * rki, rz = kz * rki;
        const double ct = clamp1((bx * kx + by * ky + bz * kz) / (rb * rk));
        const double gv = ang_g(ct), dgv = ang_dg(ct);
        const double a1 = coeff * dfck * gv, a2 = coeff * fck * dgv;
        const double fx = a1 * rx + a2 * ((ux - ct * rx) * rki);
        const double fy = a1 * ry + a2 * ((uy - ct * ry) * rki);
        const double fz = a1 * rz + a2 * ((uz - ct * rz) * rki);
        atomic_add3(F, k, fx, fy, fz);
        fcx -= fx; fcy -= fy; fcz -= fz;
    }
    atomic_add3(F, c, fcx, fcy, fcz);
}

// Four threads per atom share its row (slots jn, jn+4, jn+8): a fullerene
// atom has three bonds, so one bond per thread; this gives ~4x the
// parallelism of one thread per atom for the latency-bound bond work.
constexpr int kReboLanes = 4;

__global__ void __launch_bounds__(128)
k_rebo(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ cnt,
       const int* __restrict__ list, int cap, int na, double* __restrict__ F, double* __restrict__ part,
       const int* __restrict__ gate, int want) {
    // Gated launch (learned REBO term): runs only when *gate == want; the
    // decision is uniform over the grid, so no partial is written otherwise.
    if (gate != nullptr && *gate != want) return;
    __shared__ double sm[32 * kNV];
    double h[9], hi[9];
    load_cell(hh, h, hi);
    double acc[kNV];
#pragma unroll
    for (int k = 0; k < kNV; k++) acc[k] = 0.0;
    const long long total = (long long)na * kReboLanes;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / kReboLanes), lane = (int)(t % kReboLanes);
        const int m = cnt[i];
        double fix = 0.0, fiy = 0.0, fiz = 0.0;
        for (int jn = lane; jn < m; jn += kReboLanes) {
            const int j = list[(size_t)i * cap + jn];
            if (j <= i) continue;
            double dx, dy, dz;
            bond_vec(pos, i, j, h, hi, dx, dy, dz);
            const double rij = sqrt(norm2_rn(dx, dy, dz));
            if (rij > DMAX_CC) continue;
            const double fcut = sw_fc(rij), dfcut = sw_dfc(rij);
            if (fcut < 1e-15 && dfcut == 0) continue;
            // V_R, V_A and derivatives (AI:173-183)
            const double ea = A_CC * exp(-ALPHA_CC * rij);
            const double vr = (1.0 + Q_CC / rij) * ea;
            const double dvr = (-Q_CC / (rij * rij)) * ea + (1.0 + Q_CC / rij) * (-ALPHA_CC) * ea;
            const double e1 = exp(-BETA1_CC * rij), e2 = exp(-BETA2_CC * rij), e3 = exp(-BETA3_CC * rij);
            const double va = B1_CC * e1 + B2_CC * e2 + B3_CC * e3;
            const double dva = -BETA1_CC * B1_CC * e1 - BETA2_CC * B2_CC * e2 - BETA3_CC * B3_CC * e3;
            const double rinv = 1.0 / rij;
            const double ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;
            const double gij = bo_sum(pos, cnt, list, cap, h, hi, i, j, dx, dy, dz, rij);
            const double gji = bo_sum(pos, cnt, list, cap, h, hi, j, i, -dx, -dy, -dz, rij);
            // (1+g)^-1/2 (AI:310, 323) as a reciprocal square root
            const double bij = 1.0 / sqrt(1.0 + gij), bji = 1.0 / sqrt(1.0 + gji);
            const double bbar = 0.5 * (bij + bji);
            acc[0] += fcut * (vr - bbar * va);
            const double fpair = (dfcut * (vr - bbar * va) + fcut * (dvr - bbar * dva)) * rinv;
            fix += fpair * dx; fiy += fpair * dy; fiz += fpair * dz;
            atomic_add3(F, j, -fpair * dx, -fpair * dy, -fpair * dz);
            const double d[3] = {dx, dy, dz};
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) acc[1 + a * 3 + b] -= d[a] * fpair * d[b];
            bo_three_body(F, pos, cnt, list, cap, h, hi, i, j, dx, dy, dz, rij, ux, uy, uz, gij, bij, fcut, va);
            bo_three_body(F, pos, cnt, list, cap, h, hi, j, i, -dx, -dy, -dz, rij, -ux, -uy, -uz, gji, bji, fcut,
                          va);
        }
        if (fix != 0.0 || fiy != 0.0 || fiz != 0.0) atomic_add3(F, i, fix, fiy, fiz);
    }
    block_sum_store<kNV>(acc, sm, part + (size_t)blockIdx.x * kNV);
}

struct LJP {
    double sig2, c4, c24, rc2, vshift;
};

// Reference constants, computed with the reference's expressions.
LJP lj_params(int ff) {
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
__device__ __forceinline__ double mimg1(double d, double hii, double hii_inv) {
    double s = __dmul_rn(hii_inv, d);
    s = __dsub_rn(s, round(s));
    return __dmul_rn(hii, s);
}

template <bool FULL_VIRIAL, bool COUNT>
__device__ __forceinline__ void lj_pair(const double* __restrict__ pos, int j, double px, double py,
                                        double pz, const double* h, const double* hi, bool diag, const LJP& p,
                                        double& fx, double& fy, double& fz, double* acc) {
    double dx = __dsub_rn(pos[3 * j], px), dy = __dsub_rn(pos[3 * j + 1], py), dz = __dsub_rn(pos[3 * j + 2], pz);
    if (diag) {
        dx = mimg1(dx, h[0], hi[0]);
        dy = mimg1(dy, h[4], hi[4]);
        dz = mimg1(dz, h[8], hi[8]);
    } else {
        mimg(dx, dy, dz, hi, h);
    }
    double r2 = norm2_rn(dx, dy, dz);
    if (r2 > p.rc2) return;
    if (r2 < 0.25) r2 = 0.25;
    const double ri2 = 1.0 / r2, s2 = p.sig2 * ri2, s6 = s2 * s2 * s2, s12 = s6 * s6;
    const double fm = p.c24 * (2 * s12 - s6) * ri2;
    fx -= fm * dx; fy -= fm * dy; fz -= fm * dz;
    if (COUNT) {
        acc[0] += p.c4 * (s12 - s6) - p.vshift;
        if (FULL_VIRIAL) {
            const double d[3] = {dx, dy, dz};
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) acc[1 + a * 3 + b] += d[a] * fm * d[b];
        } else {
            acc[1] += dx * fm * dx;
            acc[5] += dy * fm * dy;
            acc[9] += dz * fm * dz;
        }
    }
}

template <bool FULL_VIRIAL>
__global__ void __launch_bounds__(256, 3)
k_lj_gather(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ cnt,
            const int* __restrict__ list, int cap, const int* __restrict__ in_cnt,
            const int* __restrict__ in_list, int in_cap, int na, double* __restrict__ F,
            double* __restrict__ Facc, LJP p, double* __restrict__ part) {
    __shared__ double sm[32 * kNV];
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    double h[9], hi[9];
    load_cell(hh, h, hi);
    // Diagonal cell (FCC/BCC boxes under the diagonal barostat): uniform branch.
    const bool diag = h[1] == 0.0 && h[2] == 0.0 && h[3] == 0.0 && h[5] == 0.0 && h[6] == 0.0 && h[7] == 0.0 &&
                      hi[1] == 0.0 && hi[2] == 0.0 && hi[3] == 0.0 && hi[5] == 0.0 && hi[6] == 0.0 && hi[7] == 0.0;
    double acc[kNV];
#pragma unroll
    for (int k = 0; k < kNV; k++) acc[k] = 0.0;
    for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < na; i += gridDim.x * wpb) {
        const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
        double fx = 0.0, fy = 0.0, fz = 0.0;
        const int m = cnt[i];
        const int* row = list + (size_t)i * cap;
        for (int k = lane; k < m; k += 32)
            lj_pair<FULL_VIRIAL, true>(pos, row[k], px, py, pz, h, hi, diag, p, fx, fy, fz, acc);
        int mi = in_cnt[i];
        mi = mi < in_cap ? mi : in_cap;
        const int* irow = in_list + (size_t)i * in_cap;
        for (int k = lane; k < mi; k += 32)
            lj_pair<FULL_VIRIAL, false>(pos, irow[k], px, py, pz, h, hi, diag, p, fx, fy, fz, acc);
        fx = warp_sum(fx); fy = warp_sum(fy); fz = warp_sum(fz);
        if (lane == 0) {
            F[3 * i] = Facc[3 * i] + fx;
            F[3 * i + 1] = Facc[3 * i + 1] + fy;
            F[3 * i + 2] = Facc[3 * i + 2] + fz;
            if (Facc != F) { Facc[3 * i] = 0.0; Facc[3 * i + 1] = 0.0; Facc[3 * i + 2] = 0.0; }
        }
    }
    block_sum_store<kNV>(acc, sm, part + (size_t)blockIdx.x * kNV);
}

__global__ void k_reduce(const double* __restrict__ part, int nblk, int nv, double* __restrict__ out) {
    __shared__ double sm[32 * 16];
    double acc[16];
#pragma unroll
    for (int k = 0; k < 16; k++) acc[k] = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
        for (int k = 0; k < nv; k++) acc[k] += part[(size_t)b * nv + k];
    double tot[16];
    block_sum_store<16>(acc, sm, tot);
    if (threadIdx.x == 0)
        for (int k = 0; k < nv; k++) out[k] = tot[k];
}

}  // namespace

cudaError_t rebo_launch(const double* pos, const double* hh, const int* cnt, const int* list, int cap,
                        int na, double* F, double* part, cudaStream_t st) {
    k_rebo<<<kForceBlocks, 128, 0, st>>>(pos, hh, cnt, list, cap, na, F, part, nullptr, 0);
    return cudaGetLastError();
}

cudaError_t rebo_launch_grid(const double* pos, const double* hh, const int* cnt, const int* list, int cap,
                             int na, double* F, double* part, int nblocks, cudaStream_t st) {
    k_rebo<<<nblocks, 128, 0, st>>>(pos, hh, cnt, list, cap, na, F, part, nullptr, 0);
    return cudaGetLastError();
}

cudaError_t rebo_launch_gated(const double* pos, const double* hh, const int* cnt, const int* list, int cap,
                              int na, double* F, double* part, int nblocks, const int* gate, int want,
                              cudaStream_t st) {
    k_rebo<<<nblocks, 128, 0, st>>>(pos, hh, cnt, list, cap, na, F, part, gate, want);
    return cudaGetLastError();
}

cudaError_t lj_gather_launch(int ff, const double* pos, const double* hh, const int* cnt, const int* list,
                             int cap, const int* in_cnt, const int* in_list, int in_cap, int na, double* F,
                             double* Facc, double* part, cudaStream_t st) {
    const LJP p = lj_params(ff);
    if (ff == FMD_FF_AIREBO)
        k_lj_gather<true><<<kForceBlocks, 256, 0, st>>>(pos, hh, cnt, list, cap, in_cnt, in_list, in_cap, na, F, Facc, p, part);
    else
        k_lj_gather<false><<<kForceBlocks, 256, 0, st>>>(pos, hh, cnt, list, cap, in_cnt, in_list, in_cap, na, F, Facc, p, part);
    return cudaGetLastError();
}

cudaError_t reduce_partials(const double* part, int nblk, int nv, double* out, cudaStream_t st) {
    k_reduce<<<1, 256, 0, st>>>(part, nblk, nv, out);
    return cudaGetLastError();
}

}  // namespace fmd
