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
#include <algorithm>
#include <cmath>
#include <map>
#include "kernels.h"
#include "geom.cuh"
#include "ljpair.cuh"
#include "ljprune.cuh"
#include "rebo_fn.cuh"
#include "step.h"
#include "umma.cuh"
#include "pdl.cuh"

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

// ------------------------------------------------- REBO on slot records --
// The fast REBO path precomputes, once per step, the geometry of every
// occupied REBO list slot (i, jn): the minimum-image bond vector d, r, 1/r,
// f_c(r) and f_c'(r).  The bond kernel then reads these records instead of
// recomputing each neighbour's image, square root and divisions for every
// bond it takes part in (each slot is used by up to 4 (cap-1) bond terms).
// The arithmetic is the reference's (AI:275-421) with cos = (d_a.d_b)/(r_a r_b)
// evaluated as (d_a.d_b) (1/r_a)(1/r_b) and one reciprocal shared by G and G'.
struct Slot {
    double dx, dy, dz, r, rinv, fc, dfc, pad;
};

__global__ void __launch_bounds__(256)
k_rebo_slots(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ cnt,
             const int* __restrict__ list, int cap, int na, Slot* __restrict__ sl,
             const int* __restrict__ gate, int want, const int* __restrict__ ids) {
    FMD_PDL_WAIT();
    if (gate != nullptr && *gate != want) return;
    __shared__ double s_hh[18];
    if (threadIdx.x < 18) s_hh[threadIdx.x] = hh[threadIdx.x];
    __syncthreads();
    const int tot = ids ? ids[0] : na * cap;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += gridDim.x * blockDim.x) {
        const int t = ids ? ids[1 + k] : k;
        if (t < 0) continue;
        const int i = t / cap, jn = t - i * cap;
        if (jn >= cnt[i]) continue;
        double x, y, z;
        bond_vec(pos, i, list[t], s_hh, s_hh + 9, x, y, z);
        const double r = sqrt(norm2_rn(x, y, z));
        Slot q;
        q.dx = x; q.dy = y; q.dz = z; q.r = r; q.rinv = 1.0 / r;
        // r > DMAX_CC is skipped by every use (AI:304, 370); f_c = 0 there.
        q.fc = r > DMAX_CC ? 0.0 : sw_fc(r);
        q.dfc = r > DMAX_CC ? 0.0 : sw_dfc(r);
        q.pad = 0.0;
        sl[t] = q;
    }
}

__device__ __forceinline__ void ang_g_dg(double x, double& g, double& dg) {
    const double c2 = G_C0 * G_C0, d2 = G_D0 * G_D0, hh = 1.0 + x, inv = 1.0 / (d2 + hh * hh);
    g = G_A0 * (1.0 + c2 / d2 - c2 * inv);
    dg = G_A0 * 2.0 * c2 * hh * inv * inv;
}

// Sum over centre c's other slots of f_c G(cos) for the bond in slot skip_kn
// of c's row (-1: the bond is not in c's row) whose vector is s*(bx,by,bz)
// with s = +-1 (AI:301-309).  Rows hold no atom twice, so skipping the slot is
// skipping the bonded atom.
__device__ __forceinline__ double bo_sum_sl(const Slot* __restrict__ sl, int cap, int c, int m, int skip_kn,
                                            double bx, double by, double bz, double rbinv) {
    double gs = 0.0;
    for (int kn = 0; kn < m; kn++) {
        const size_t o = (size_t)c * cap + kn;
        if (kn == skip_kn) continue;
        const Slot q = sl[o];
        if (q.fc < 1e-15) continue;
        const double ct = clamp1((bx * q.dx + by * q.dy + bz * q.dz) * (rbinv * q.rinv));
        double g, dg;
        ang_g_dg(ct, g, dg);
        gs += q.fc * g;
    }
    return gs;
}

// Bond order of every directed slot c -> j (AI:301-323 for centre c):
// g = sum over c's other slots of f_c G(cos), b = (1 + g)^-1/2, the pair
// functions of r_cj (AI:173-183) and the three-body coefficient
// coeff = -(f_c V_A / 2) db/dg (AI:361-365; zero where the reference skips
// the three-body block).  bo[t] = {b, g, coeff, vr, dvr, va, dva, ok}.
struct SlotBO {
    double b, g, coeff, vr, dvr, va, dva, ok;
};

__device__ __forceinline__ void rebo_pair_fn(double r, double rinv, double& vr, double& dvr, double& va,
                                             double& dva) {
    const double ea = A_CC * exp(-ALPHA_CC * r);
    const double qr = Q_CC * rinv;
    vr = (1.0 + qr) * ea;
    dvr = (-qr * rinv) * ea + (1.0 + qr) * (-ALPHA_CC) * ea;
    const double e1 = exp(-BETA1_CC * r), e2 = exp(-BETA2_CC * r), e3 = exp(-BETA3_CC * r);
    va = B1_CC * e1 + B2_CC * e2 + B3_CC * e3;
    dva = -BETA1_CC * B1_CC * e1 - BETA2_CC * B2_CC * e2 - BETA3_CC * B3_CC * e3;
}

// Three-body coefficient of centre c for a bond with f_c and V_A.
__device__ __forceinline__ double three_body_coeff(double gs, double b, double fcut, double va) {
    if (!(fabs(gs) > 1e-20 && va > 1e-20)) return 0.0;
    const double dbp = -BO_DELTA * b / (1.0 + gs);
    return -(0.5 * fcut * va) * dbp;
}

__global__ void __launch_bounds__(256)
k_rebo_bo(const Slot* __restrict__ sl, const int* __restrict__ cnt, const int* __restrict__ list, int cap, int na,
          SlotBO* __restrict__ bo, const int* __restrict__ gate, int want, const int* __restrict__ ids) {
    FMD_PDL_WAIT();
    if (gate != nullptr && *gate != want) return;
    const int tot = ids ? ids[0] : na * cap;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += gridDim.x * blockDim.x) {
        const int t = ids ? ids[1 + k] : k;
        if (t < 0) continue;
        const int c = t / cap, jn = t - c * cap;
        const int m = cnt[c];
        if (jn >= m) continue;
        const Slot q = sl[t];
        SlotBO o;
        o.ok = 0.0;
        // the reference's bond gate (AI:292-296)
        if (q.r <= DMAX_CC && !(q.fc < 1e-15 && q.dfc == 0)) {
            const double g = bo_sum_sl(sl, cap, c, m, jn, q.dx, q.dy, q.dz, q.rinv);
            o.g = g;
            o.b = 1.0 / sqrt(1.0 + g);
            rebo_pair_fn(q.r, q.rinv, o.vr, o.dvr, o.va, o.dva);
            o.coeff = three_body_coeff(g, o.b, q.fc, o.va);
            o.ok = 1.0;
        }
        bo[t] = o;
    }
}

// Slot geometry and bond order in one pass over the warp-aligned slot index
// (the slots of one centre are consecutive lanes of one warp): each lane
// computes its own slot's record (as k_rebo_slots), then takes the other
// slots' vectors from their lanes by shuffles and sums f_c G(cos) in slot
// order (as bo_sum_sl), so the bond order needs no slot-record reads and
// both records come out bit for bit as the two-kernel path writes them.
__global__ void __launch_bounds__(256)
k_rebo_geo_bo(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ cnt,
              const int* __restrict__ list, int cap, Slot* __restrict__ sl, SlotBO* __restrict__ bo,
              const int* __restrict__ gate, int want, const int* __restrict__ ids) {
    FMD_PDL_WAIT();
    if (gate != nullptr && *gate != want) return;
    __shared__ double s_hh[18];
    if (threadIdx.x < 18) s_hh[threadIdx.x] = hh[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int tot = ids[0];
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < tot; base += gridDim.x * blockDim.x) {
        const int k = base + lane;
        int t = k < tot ? ids[1 + k] : -1;
        const bool valid = t >= 0;
        if (!valid) t = 0;
        const int c = t / cap, jn = t - c * cap;
        const int m = valid ? cnt[c] : 0;
        Slot q;
        q.dx = q.dy = q.dz = q.r = q.fc = q.dfc = q.pad = 0.0;
        q.rinv = 0.0;
        if (valid) {
            double x, y, z;
            bond_vec(pos, c, list[t], s_hh, s_hh + 9, x, y, z);
            const double r = sqrt(norm2_rn(x, y, z));
            q.dx = x; q.dy = y; q.dz = z; q.r = r; q.rinv = 1.0 / r;
            // r > DMAX_CC is skipped by every use (AI:304, 370); f_c = 0 there.
            q.fc = r > DMAX_CC ? 0.0 : sw_fc(r);
            q.dfc = r > DMAX_CC ? 0.0 : sw_dfc(r);
            sl[t] = q;
        }
        const unsigned seg = __match_any_sync(kFull, valid ? c : -1 - lane);
        const int s0 = __ffs(seg) - 1;
        const int span = (int)__reduce_max_sync(kFull, (unsigned)m);
        // the reference's bond gate (AI:292-296)
        const bool need = valid && q.r <= DMAX_CC && !(q.fc < 1e-15 && q.dfc == 0);
        double gs = 0.0;
        for (int kn = 0; kn < span; kn++) {
            const int src = s0 + (kn < m ? kn : 0);
            const double kx = __shfl_sync(kFull, q.dx, src), ky = __shfl_sync(kFull, q.dy, src),
                         kz = __shfl_sync(kFull, q.dz, src), kri = __shfl_sync(kFull, q.rinv, src),
                         kfc = __shfl_sync(kFull, q.fc, src);
            if (need && kn < m && kn != jn && !(kfc < 1e-15)) {
                const double ct = clamp1((q.dx * kx + q.dy * ky + q.dz * kz) * (q.rinv * kri));
                double g, dg;
                ang_g_dg(ct, g, dg);
                gs += kfc * g;
            }
        }
        if (valid) {
            SlotBO o;
            o.b = o.g = o.coeff = o.vr = o.dvr = o.va = o.dva = 0.0;
            o.ok = 0.0;
            if (need) {
                o.g = gs;
                o.b = 1.0 / sqrt(1.0 + gs);
                rebo_pair_fn(q.r, q.rinv, o.vr, o.dvr, o.va, o.dva);
                o.coeff = three_body_coeff(gs, o.b, q.fc, o.va);
                o.ok = 1.0;
            }
            bo[t] = o;
        }
    }
}

// Three-body forces of centre c for the bond c -> skip with coefficient coeff
// (AI:368-419) on c's other neighbours k, and the reaction on c.
// PHYS: the gradient of the bond-order term instead of the reference's
// three-body forces (which have the opposite sign on the neighbours and lack
// the term on the bond partner): f_k = -coeff dG/dr_k, and the partner gets
// -coeff dG/dr_skip = -coeff sum_k fc_k g'(cos) (u_k - cos u_b) / r_b.
template <bool PHYS>
__device__ __forceinline__ void three_body_sl(double* __restrict__ F, const Slot* __restrict__ sl,
                                              const int* __restrict__ list, int cap, int c, int m, int skip,
                                              double bx, double by, double bz, double rbinv, double coeff) {
    if (coeff == 0.0) return;
    const double ux = bx * rbinv, uy = by * rbinv, uz = bz * rbinv;
    double fcx = 0.0, fcy = 0.0, fcz = 0.0;
    double fbx = 0.0, fby = 0.0, fbz = 0.0;
    for (int kn = 0; kn < m; kn++) {
        const size_t o = (size_t)c * cap + kn;
        const int k = list[o];
        if (k == skip) continue;
        const Slot q = sl[o];
        if (q.fc < 1e-15) continue;
        const double rx = q.dx * q.rinv, ry = q.dy * q.rinv, rz = q.dz * q.rinv;
        const double ct = clamp1((bx * q.dx + by * q.dy + bz * q.dz) * (rbinv * q.rinv));
        double gv, dgv;
        ang_g_dg(ct, gv, dgv);
        const double a1 = PHYS ? -(coeff * q.dfc * gv) : coeff * q.dfc * gv;
        const double a2 = PHYS ? -(coeff * q.fc * dgv) : coeff * q.fc * dgv;
        const double fx = a1 * rx + a2 * ((ux - ct * rx) * q.rinv);
        const double fy = a1 * ry + a2 * ((uy - ct * ry) * q.rinv);
        const double fz = a1 * rz + a2 * ((uz - ct * rz) * q.rinv);
        atomic_add3(F, k, fx, fy, fz);
        fcx -= fx; fcy -= fy; fcz -= fz;
        if (PHYS) {
            const double a3 = a2 * rbinv;
            fbx += a3 * (rx - ct * ux); fby += a3 * (ry - ct * uy); fbz += a3 * (rz - ct * uz);
        }
    }
    if (PHYS) {
        atomic_add3(F, skip, fbx, fby, fbz);
        fcx -= fbx; fcy -= fby; fcz -= fbz;
    }
    atomic_add3(F, c, fcx, fcy, fcz);
}

// Sum of (x, y, z) over the lanes of this lane's segment, left in the segment's
// lowest lane.  Segments are runs of consecutive lanes (seg: this lane's
// segment as a lane mask, span: the longest segment of the warp); lane L ends
// with the sum over L .. its segment's last lane, so the lowest lane holds
// the whole sum.  Fixed order.
__device__ __forceinline__ void seg_sum3(double& x, double& y, double& z, unsigned seg, int lane, int span) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        if (o >= span) break;                          // uniform over the warp
        const double wx = __shfl_down_sync(kFull, x, o);
        const double wy = __shfl_down_sync(kFull, y, o);
        const double wz = __shfl_down_sync(kFull, z, o);
        if (lane + o < 32 && ((seg >> (lane + o)) & 1u)) { x += wx; y += wy; z += wz; }
    }
}

// Forces, one lane per directed slot i -> j.  The reference enumerates
// bonds from the row of the lower index (AI:288) and evaluates the three-body
// blocks of both ends from their own rows.  Here the slot i -> j does the
// three-body block of centre i, and for j > i also the pair term; when the
// list is asymmetric (rows truncated at cap) and j's row lacks i, the owning
// slot (j > i) also computes b_ji and centre j's block from j's row, and a
// slot with j < i whose partner is missing does nothing (the reference never
// visits that bond).
//
// The slots of one centre sit in consecutive lanes (atom-major slot order),
// and at step kn of the three-body loop every one of them pushes a force onto
// the same neighbour list[i][kn]: the lanes of the centre sum it first
// (seg_sum) and one lane adds it, and the reactions on the centre and its
// pair-term forces go out as one sum per centre, so a centre with m bonds
// issues about m + 1 + m/2 atomic triples instead of m^2 + m/2.
template <bool PHYS>
__global__ void __launch_bounds__(256)
k_rebo_force(const Slot* __restrict__ sl, const SlotBO* __restrict__ bo, const int* __restrict__ cnt,
             const int* __restrict__ list, int cap, int na, double* __restrict__ F, double* __restrict__ part,
             const int* __restrict__ gate, int want, const int* __restrict__ ids) {
    FMD_PDL_WAIT();
    if (gate != nullptr && *gate != want) return;
    __shared__ double sm[32 * kNV];
    double acc[kNV];
#pragma unroll
    for (int k = 0; k < kNV; k++) acc[k] = 0.0;
    const int lane = threadIdx.x & 31;
    const int tot = ids ? ids[0] : na * cap;
    // warp-uniform loop: the shuffles below need every lane
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < tot; base += gridDim.x * blockDim.x) {
        const int kk = base + lane;
        bool valid = kk < tot;
        int t = valid ? (ids ? ids[1 + kk] : kk) : 0;
        if (t < 0) { valid = false; t = 0; }            // padding lane of the slot index
        const int i = t / cap, jn = t - i * cap;
        const int m = valid ? cnt[i] : 0;
        valid = valid && jn < m;
        bool ok = false;
        SlotBO o;
        o.b = o.g = o.coeff = o.vr = o.dvr = o.va = o.dva = o.ok = 0.0;
        if (valid) {
            o = bo[t];
            ok = o.ok != 0.0;
        }
        int j = -1, pn = -1, mj = 0;
        if (ok) {
            j = list[t];
            mj = cnt[j];
            if (ids) {
                pn = ids[1 + (size_t)kIdsLanes * na + t];   // partner slot j -> i of the last build
            } else {
                for (int kn = 0; kn < mj; kn++)
                    if (list[(size_t)j * cap + kn] == i) { pn = kn; break; }
            }
            if (j < i && pn < 0) ok = false;
        }
        Slot q;
        q.dx = q.dy = q.dz = q.r = q.rinv = q.fc = q.dfc = q.pad = 0.0;
        if (ok) q = sl[t];
        // lanes of one centre (a lane that is not a slot is alone)
        const unsigned seg = __match_any_sync(kFull, valid ? i : -1 - lane);
        const bool lead = lane == __ffs(seg) - 1;
        const int span = __reduce_max_sync(kFull, (unsigned)__popc(seg));
        double fcx = 0.0, fcy = 0.0, fcz = 0.0;      // force on the centre i from this slot
        // three-body block of centre i for the bond i -> j (AI:368-419)
        const bool tb = ok && o.coeff != 0.0;
        const double ux = q.dx * q.rinv, uy = q.dy * q.rinv, uz = q.dz * q.rinv;
        const int mseg = __reduce_max_sync(kFull, valid ? m : 0);
        double fbx = 0.0, fby = 0.0, fbz = 0.0;       // PHYS: force on the partner j
        for (int kn = 0; kn < mseg; kn++) {
            double fx = 0.0, fy = 0.0, fz = 0.0;
            int kt = -1;
            if (valid && kn < m) {
                const size_t off = (size_t)i * cap + kn;
                kt = list[off];
                if (tb && kt != j) {
                    const Slot r = sl[off];
                    if (!(r.fc < 1e-15)) {
                        const double rx = r.dx * r.rinv, ry = r.dy * r.rinv, rz = r.dz * r.rinv;
                        const double ct = clamp1((q.dx * r.dx + q.dy * r.dy + q.dz * r.dz) * (q.rinv * r.rinv));
                        double gv, dgv;
                        ang_g_dg(ct, gv, dgv);
                        const double a1 = PHYS ? -(o.coeff * r.dfc * gv) : o.coeff * r.dfc * gv;
                        const double a2 = PHYS ? -(o.coeff * r.fc * dgv) : o.coeff * r.fc * dgv;
                        fx = a1 * rx + a2 * ((ux - ct * rx) * r.rinv);
                        fy = a1 * ry + a2 * ((uy - ct * ry) * r.rinv);
                        fz = a1 * rz + a2 * ((uz - ct * rz) * r.rinv);
                        fcx -= fx; fcy -= fy; fcz -= fz;
                        if (PHYS) {
                            const double a3 = a2 * q.rinv;
                            fbx += a3 * (rx - ct * ux); fby += a3 * (ry - ct * uy); fbz += a3 * (rz - ct * uz);
                        }
                    }
                }
            }
            seg_sum3(fx, fy, fz, seg, lane, span);
            if (lead && kt >= 0 && (fx != 0.0 || fy != 0.0 || fz != 0.0)) atomic_add3(F, kt, fx, fy, fz);
        }
        if (PHYS && tb) {
            atomic_add3(F, j, fbx, fby, fbz);
            fcx -= fbx; fcy -= fby; fcz -= fbz;
        }
        if (ok && j > i) {
            double bji;
            if (pn >= 0) {
                bji = bo[(size_t)j * cap + pn].b;
            } else {
                const double gji = bo_sum_sl(sl, cap, j, mj, -1, -q.dx, -q.dy, -q.dz, q.rinv);
                bji = 1.0 / sqrt(1.0 + gji);
                three_body_sl<PHYS>(F, sl, list, cap, j, mj, i, -q.dx, -q.dy, -q.dz, q.rinv,
                                    three_body_coeff(gji, bji, q.fc, o.va));
            }
            const double bbar = 0.5 * (o.b + bji);
            acc[0] += q.fc * (o.vr - bbar * o.va);
            const double fpair = (q.dfc * (o.vr - bbar * o.va) + q.fc * (o.dvr - bbar * o.dva)) * q.rinv;
            fcx += fpair * q.dx; fcy += fpair * q.dy; fcz += fpair * q.dz;
            atomic_add3(F, j, -fpair * q.dx, -fpair * q.dy, -fpair * q.dz);
            const double d[3] = {q.dx, q.dy, q.dz};
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) acc[1 + a * 3 + b] -= d[a] * fpair * d[b];
        }
        seg_sum3(fcx, fcy, fcz, seg, lane, span);
        if (lead && valid && (fcx != 0.0 || fcy != 0.0 || fcz != 0.0)) atomic_add3(F, i, fcx, fcy, fcz);
    }
    block_sum_store<kNV>(acc, sm, part + (size_t)blockIdx.x * kNV);
}

LJP lj_params(int ff) { return lj_params_dev(ff); }

// Entries per lane in flight (U): the index loads of U entries are issued
// together, then their positions, then the pair arithmetic, so one warp has
// U dependent load chains outstanding instead of one.  PIPE additionally
// software-pipelines the lane's loop: the indices and positions of the next
// U entries are loaded before the current U are computed, so their latency
// overlaps the arithmetic.
template <int U>
__device__ __forceinline__ void lj_fetch(const double* __restrict__ pos, const int* __restrict__ row, int tot,
                                         int b, int i, int (&jj)[U], double (&qx)[U], double (&qy)[U],
                                         double (&qz)[U]) {
#pragma unroll
    for (int u = 0; u < U; u++) {
        const int k = b + 32 * u;
        jj[u] = k < tot ? row[k] : -1;
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
        const int j = jj[u] < 0 ? i : jj[u];
        qx[u] = pos[3 * j]; qy[u] = pos[3 * j + 1]; qz[u] = pos[3 * j + 2];
    }
}

// Pair terms of one chunk (U entries per lane; jc < 0: none) seen from atom i.
// A pruning gather (po.cnt set) also appends the chunk's entries with
// r^2 <= po.r2 to prow in row order (entry b0 + 32 u + lane, u then lane
// ascending); every lane of the warp must call this.
template <bool FULL_VIRIAL, bool F32, int U>
__device__ __forceinline__ void lj_chunk(const int (&jc)[U], const double (&cx)[U], const double (&cy)[U],
                                         const double (&cz)[U], int i, double px, double py, double pz,
                                         const double* h, const double* hi, bool diag, bool wide, const LJP& p,
                                         const LJF& pf,
                                         double& fx, double& fy, double& fz, double* acc, const LJPruneOut& po,
                                         int* __restrict__ prow, int& pc, int lane) {
    bool keep[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
        keep[u] = false;
        if (jc[u] < 0) continue;
        double dx = __dsub_rn(cx[u], px), dy = __dsub_rn(cy[u], py), dz = __dsub_rn(cz[u], pz);
        if (wide) {
            dx = mimg1_rint(dx, h[0], hi[0]);
            dy = mimg1_rint(dy, h[4], hi[4]);
            dz = mimg1_rint(dz, h[8], hi[8]);
        } else if (diag) {
            dx = mimg1(dx, h[0], hi[0]);
            dy = mimg1(dy, h[4], hi[4]);
            dz = mimg1(dz, h[8], hi[8]);
        } else {
            mimg(dx, dy, dz, hi, h);
        }
        if (po.cnt) keep[u] = norm2_rn(dx, dy, dz) <= po.r2;
        if (jc[u] > i) lj_pair<FULL_VIRIAL, F32, true>(dx, dy, dz, p, pf, fx, fy, fz, acc);
        else lj_pair<FULL_VIRIAL, F32, false>(dx, dy, dz, p, pf, fx, fy, fz, acc);
    }
    if (po.cnt) {
#pragma unroll
        for (int u = 0; u < U; u++) {
            const unsigned m = __ballot_sync(kFull, keep[u]);
            if (keep[u]) prow[pc + __popc(m & ((1u << lane) - 1u))] = jc[u];
            pc += __popc(m);
        }
    }
}

// Facc[i] for lj_atom_done, read by lane 0 when the atom's row starts so the
// load is not on the row's tail.
struct LJAcc {
    double x = 0.0, y = 0.0, z = 0.0;
};
__device__ __forceinline__ LJAcc lj_acc_load(const double* __restrict__ Facc, int i, int lane) {
    LJAcc a;
    if (lane == 0) { a.x = Facc[3 * i]; a.y = Facc[3 * i + 1]; a.z = Facc[3 * i + 2]; }
    return a;
}

// End of atom i's row: F[i] = Facc[i] (fa, read at the row's start) + the
// warp's sum (Facc cleared), and for a pruning gather the pruned row's length
// and i's fractional position.
__device__ __forceinline__ void lj_atom_done(int i, double fx, double fy, double fz, double px, double py,
                                             double pz, const double* hi, double* __restrict__ F,
                                             double* __restrict__ Facc, const LJPruneOut& po, int pc, int lane,
                                             const LJAcc& fa) {
    fx = warp_sum(fx); fy = warp_sum(fy); fz = warp_sum(fz);
    if (lane == 0) {
        F[3 * i] = fa.x + fx;
        F[3 * i + 1] = fa.y + fy;
        F[3 * i + 2] = fa.z + fz;
        if (Facc != F) { Facc[3 * i] = 0.0; Facc[3 * i + 1] = 0.0; Facc[3 * i + 2] = 0.0; }
        if (po.cnt) {
            po.cnt[i] = pc;
            po.sb[3 * i] = hi[0] * px + hi[1] * py + hi[2] * pz;
            po.sb[3 * i + 1] = hi[3] * px + hi[4] * py + hi[5] * pz;
            po.sb[3 * i + 2] = hi[6] * px + hi[7] * py + hi[8] * pz;
        }
    }
}

// Atoms of warp w of block blk out of nblk blocks of W warps: strided over
// the system (i = blk W + w, step nblk W), or (contig) block blk's own run of
// consecutive atoms [blk na / nblk, (blk + 1) na / nblk), warps interleaved.
struct AtomRange {
    int first, end, step;
};
__device__ __forceinline__ AtomRange atom_range(int blk, int nblk, int W, int w, int na, bool contig) {
    if (!contig) return AtomRange{blk * W + w, na, nblk * W};
    const int a0 = (int)((long long)blk * na / nblk), a1 = (int)((long long)(blk + 1) * na / nblk);
    return AtomRange{a0 + w, a1, W};
}

// One gather pass over atoms blk, blk + nblk, ... (in warps) of one system;
// per-block {E, W9} into part[blk].  sm: 32 * kNV doubles, s_hh: 18.
// Row i of the full list (in_list, stride in_cap, in_cnt[i] entries) is the
// incoming entries (j < i, from the transposed half list) followed by the
// reference row (j > i), so a pair is counted for energy and virial on the
// side where j > i.
template <bool FULL_VIRIAL, bool F32, int U, bool PIPE>
__device__ __forceinline__ void lj_gather_body(const double* __restrict__ pos, const double* __restrict__ hh,
                                               const int* __restrict__ in_cnt, const int* __restrict__ in_list,
                                               int in_cap, int na, double* __restrict__ F,
                                               double* __restrict__ Facc, const LJP& p, double* __restrict__ part,
                                               int blk, int nblk, double* sm, double* s_hh,
                                               const LJPruneOut& po, bool contig = false) {
    if (threadIdx.x < 18) s_hh[threadIdx.x] = hh[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    const double* h = s_hh;
    const double* hi = s_hh + 9;
    // Diagonal cell (FCC/BCC boxes under the diagonal barostat): uniform branch.
    const bool diag = h[1] == 0.0 && h[2] == 0.0 && h[3] == 0.0 && h[5] == 0.0 && h[6] == 0.0 && h[7] == 0.0 &&
                      hi[1] == 0.0 && hi[2] == 0.0 && hi[3] == 0.0 && hi[5] == 0.0 && hi[6] == 0.0 && hi[7] == 0.0;
    // half the narrowest edge beyond the cutoff: the one-instruction image (mimg1_rint)
    const bool wide = diag && 0.25 * fmin(h[0] * h[0], fmin(h[4] * h[4], h[8] * h[8])) > p.rc2 * (1.0 + 1e-9);
    const LJF pf{(float)p.sig2, (float)(p.sig2 - (double)(float)p.sig2), (float)p.c4, (float)p.c24};
    double acc[kNV];
#pragma unroll
    for (int k = 0; k < kNV; k++) acc[k] = 0.0;
    const AtomRange ar = atom_range(blk, nblk, wpb, threadIdx.x >> 5, na, contig);
    for (int i = ar.first; i < ar.end; i += ar.step) {
        const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
        const LJAcc fa = lj_acc_load(Facc, i, lane);
        double fx = 0.0, fy = 0.0, fz = 0.0;
        const int tot = min(in_cnt[i], in_cap);
        const int* row = in_list + (size_t)i * in_cap;
        int* prow = po.cnt ? po.list + (size_t)i * in_cap : nullptr;
        int pc = 0;
        int jj[U];
        double qx[U], qy[U], qz[U];
        if (PIPE && tot > 0) lj_fetch<U>(pos, row, tot, lane, i, jj, qx, qy, qz);
        for (int b0 = 0; b0 < tot; b0 += 32 * U) {       // uniform over the warp
            int jc[U];
            double cx[U], cy[U], cz[U];
            if (PIPE) {
#pragma unroll
                for (int u = 0; u < U; u++) { jc[u] = jj[u]; cx[u] = qx[u]; cy[u] = qy[u]; cz[u] = qz[u]; }
                if (b0 + 32 * U < tot) lj_fetch<U>(pos, row, tot, b0 + 32 * U + lane, i, jj, qx, qy, qz);
            } else {
                lj_fetch<U>(pos, row, tot, b0 + lane, i, jc, cx, cy, cz);
            }
            lj_chunk<FULL_VIRIAL, F32, U>(jc, cx, cy, cz, i, px, py, pz, h, hi, diag, wide, p, pf, fx, fy, fz, acc, po,
                                          prow, pc, lane);
        }
        lj_atom_done(i, fx, fy, fz, px, py, pz, hi, F, Facc, po, pc, lane, fa);
    }
    lj_virial_mirror<FULL_VIRIAL>(acc);
    block_sum_store<kNV>(acc, sm, part + (size_t)blk * kNV);
}

// The rows of this evaluation: with po.words set, the full rows and pruned-
// row output when a prune is due, else the pruned rows (po.cnt, po.list) and
// no output; every block decides on the same inputs.
__device__ __forceinline__ void lj_rows_select(const double* hh, const int*& rcnt, const int*& rlist,
                                               LJPruneOut& po) {
    if (!po.words || lj_prune_needed(po.words, hh, po.hb, po.delta, po.rc)) return;
    rcnt = po.cnt;
    rlist = po.list;
    po.cnt = nullptr;
}

// Records gridDim.x .. nrec-1 of part are zero: the gathers of one system
// may run on different grids and write one record count.
__device__ __forceinline__ void lj_zero_records(double* __restrict__ part, int nrec) {
    if (threadIdx.x < kNV)
        for (int r = gridDim.x + blockIdx.x; r < nrec; r += gridDim.x) part[(size_t)r * kNV + threadIdx.x] = 0.0;
}

template <bool FULL_VIRIAL, bool F32, int U, bool PIPE, int NT>
__global__ void __launch_bounds__(NT)
k_lj_gather(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ in_cnt,
            const int* __restrict__ in_list, int in_cap, int na, double* __restrict__ F,
            double* __restrict__ Facc, LJP p, double* __restrict__ part, LJPruneOut po, int nrec, int contig) {
    FMD_PDL_WAIT();
    __shared__ double sm[32 * kNV];
    __shared__ double s_hh[18];
    const int* rcnt = in_cnt;
    const int* rlist = in_list;
    lj_rows_select(hh, rcnt, rlist, po);
    lj_gather_body<FULL_VIRIAL, F32, U, PIPE>(pos, hh, rcnt, rlist, in_cap, na, F, Facc, p, part, blockIdx.x,
                                              gridDim.x, sm, s_hh, po, contig != 0);
    lj_zero_records(part, nrec);
}

// Row-staged gather: each warp copies its next atom's full row into a
// shared-memory buffer with one bulk asynchronous copy (cp.async.bulk,
// completion on an mbarrier) while it computes the current atom from the
// other buffer, so the row stream from HBM overlaps the pair arithmetic
// instead of sitting on each iteration's dependency chain.  Requires row
// stride in_cap % 4 == 0 (16-byte aligned rows).  Every wait is bounded: on a
// timeout the kernel records K_LJ in err, waits (bounded) for its own copy in
// flight and returns.
__device__ __forceinline__ void bulk_row(int* dst, const int* src, uint32_t bytes, uint64_t* mbar) {
    const uint32_t m = umma::smem_u32(mbar), d = umma::smem_u32(dst);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(m), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(d), "l"(src), "r"(bytes), "r"(m)
                 : "memory");
}

template <bool FULL_VIRIAL, bool F32, int U, int NT>
__device__ __forceinline__ void lj_gather_staged_body(const double* __restrict__ pos, const double* __restrict__ hh,
                                                      const int* __restrict__ in_cnt, const int* __restrict__ in_list,
                                                      int in_cap, int na, double* __restrict__ F,
                                                      double* __restrict__ Facc, const LJP& p,
                                                      double* __restrict__ part, DevErr* err, int blk, int nblk,
                                                      unsigned char* dsm, double* sm, double* s_hh,
                                                      const LJPruneOut& po, bool contig = false) {
    constexpr int W = NT / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int* bufs = reinterpret_cast<int*>(dsm) + (size_t)w * 2 * in_cap;
    uint64_t* mb = reinterpret_cast<uint64_t*>(dsm + (size_t)W * 2 * in_cap * sizeof(int)) + 2 * w;
    if (lane == 0) {
        umma::mbar_init(&mb[0], 1);
        umma::mbar_init(&mb[1], 1);
    }
    if (threadIdx.x < 18) s_hh[threadIdx.x] = hh[threadIdx.x];
    __syncthreads();
    const double* h = s_hh;
    const double* hi = s_hh + 9;
    const bool diag = h[1] == 0.0 && h[2] == 0.0 && h[3] == 0.0 && h[5] == 0.0 && h[6] == 0.0 && h[7] == 0.0 &&
                      hi[1] == 0.0 && hi[2] == 0.0 && hi[3] == 0.0 && hi[5] == 0.0 && hi[6] == 0.0 && hi[7] == 0.0;
    // half the narrowest edge beyond the cutoff: the one-instruction image (mimg1_rint)
    const bool wide = diag && 0.25 * fmin(h[0] * h[0], fmin(h[4] * h[4], h[8] * h[8])) > p.rc2 * (1.0 + 1e-9);
    const LJF pf{(float)p.sig2, (float)(p.sig2 - (double)(float)p.sig2), (float)p.c4, (float)p.c24};
    double acc[kNV];
#pragma unroll
    for (int k = 0; k < kNV; k++) acc[k] = 0.0;
    auto issue = [&](int atom, int b) {
        const int nrow = min(in_cnt[atom], in_cap);
        const uint32_t bytes = (uint32_t)max(16, (nrow * 4 + 15) & ~15);
        umma::fence_smem_async();               // earlier reads of this buffer before the async write
        bulk_row(bufs + (size_t)b * in_cap, in_list + (size_t)atom * in_cap, bytes, &mb[b]);
    };
    const AtomRange ar = atom_range(blk, nblk, W, w, na, contig);
    const int stride = ar.step, iend = ar.end;
    int i = ar.first;
    uint32_t ph0 = 0, ph1 = 0;
    int cur = 0;
    bool pending = false;                       // a copy into buffer cur ^ 1 may be in flight
    if (i < iend && lane == 0) issue(i, 0);
    for (; i < iend; i += stride) {
        const int inext = i + stride;
        if (inext < iend && lane == 0) issue(inext, cur ^ 1);
        pending = inext < iend;
        const bool ok = umma::mbar_wait(&mb[cur], cur ? ph1 : ph0);
        if (cur) ph1 ^= 1; else ph0 ^= 1;
        if (!__all_sync(kFull, ok)) {
            if (lane == 0 && atomicCAS(&err->code, FMD_OK, FMD_ERR_CUDA) == FMD_OK) {
                err->where = K_LJ; err->index = i; err->value = 0;
            }
            break;
        }
        const int* row = bufs + (size_t)cur * in_cap;
        const int tot = min(in_cnt[i], in_cap);
        const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
        const LJAcc fa = lj_acc_load(Facc, i, lane);
        double fx = 0.0, fy = 0.0, fz = 0.0;
        int* prow = po.cnt ? po.list + (size_t)i * in_cap : nullptr;
        int pc = 0;
        for (int b0 = 0; b0 < tot; b0 += 32 * U) {       // uniform over the warp
            const int b = b0 + lane;
            int jc[U];
            double cx[U], cy[U], cz[U];
#pragma unroll
            for (int u = 0; u < U; u++) jc[u] = b + 32 * u < tot ? row[b + 32 * u] : -1;
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int j = jc[u] < 0 ? i : jc[u];
                cx[u] = pos[3 * j]; cy[u] = pos[3 * j + 1]; cz[u] = pos[3 * j + 2];
            }
            lj_chunk<FULL_VIRIAL, F32, U>(jc, cx, cy, cz, i, px, py, pz, h, hi, diag, wide, p, pf, fx, fy, fz, acc, po,
                                          prow, pc, lane);
        }
        lj_atom_done(i, fx, fy, fz, px, py, pz, hi, F, Facc, po, pc, lane, fa);
        __syncwarp();                           // buffer cur is reused two atoms on
        cur ^= 1;
        pending = false;
    }
    // after an early exit, the copy issued for the next atom may still be in flight
    if (pending) umma::mbar_wait(&mb[cur ^ 1], (cur ^ 1) ? ph1 : ph0);
    lj_virial_mirror<FULL_VIRIAL>(acc);
    block_sum_store<kNV>(acc, sm, part + (size_t)blk * kNV);
}

template <bool FULL_VIRIAL, bool F32, int U, int NT>
__global__ void __launch_bounds__(NT)
k_lj_gather_staged(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ in_cnt,
                   const int* __restrict__ in_list, int in_cap, int na, double* __restrict__ F,
                   double* __restrict__ Facc, LJP p, double* __restrict__ part, DevErr* err,
                   LJPruneOut po, int nrec, int contig) {
    FMD_PDL_WAIT();
    extern __shared__ __align__(128) unsigned char dsm[];
    __shared__ double sm[32 * kNV];
    __shared__ double s_hh[18];
    const int* rcnt = in_cnt;
    const int* rlist = in_list;
    lj_rows_select(hh, rcnt, rlist, po);
    lj_gather_staged_body<FULL_VIRIAL, F32, U, NT>(pos, hh, rcnt, rlist, in_cap, na, F, Facc, p, part, err,
                                                   blockIdx.x, gridDim.x, dsm, sm, s_hh, po, contig != 0);
    lj_zero_records(part, nrec);
}

// Replica batch, rows staged (all replicas share the row stride in_cap).
template <bool FULL_VIRIAL, bool F32, int U, int NT>
__global__ void __launch_bounds__(NT)
k_b_lj_gather_staged(const StepArrays* __restrict__ As, const int* __restrict__ off, int R, int ff) {
    extern __shared__ __align__(128) unsigned char dsm[];
    __shared__ double sm[32 * kNV];
    __shared__ double s_hh[18];
    const int r = batch_rep(off, R, blockIdx.x);
    const StepArrays& a = As[r];
    const LJP p = lj_params_dev(ff);
    lj_gather_staged_body<FULL_VIRIAL, F32, U, NT>(a.pos, a.S->h, a.in_cnt, a.in_list, a.in_cap, a.n, a.F, a.Facc, p,
                                                   a.part_f2, a.err, blockIdx.x - off[r], off[r + 1] - off[r], dsm,
                                                   sm, s_hh, LJPruneOut{});
}

// Replica batch: the same gather over every replica in one launch; block b
// serves replica r = batch_rep(off, R, b) as its local block b - off[r].
template <bool FULL_VIRIAL, bool F32, int U, int NT>
__global__ void __launch_bounds__(NT)
k_b_lj_gather(const StepArrays* __restrict__ As, const int* __restrict__ off, int R, int ff) {
    __shared__ double sm[32 * kNV];
    __shared__ double s_hh[18];
    const int r = batch_rep(off, R, blockIdx.x);
    const StepArrays& a = As[r];
    const LJP p = lj_params_dev(ff);
    lj_gather_body<FULL_VIRIAL, F32, U, false>(a.pos, a.S->h, a.in_cnt, a.in_list, a.in_cap,
                                        a.n, a.F, a.Facc, p, a.part_f2, blockIdx.x - off[r], off[r + 1] - off[r], sm,
                                        s_hh, LJPruneOut{});
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

cudaError_t rebo_slots_launch(const double* pos, const double* hh, const int* cnt, const int* list, int cap,
                              int na, double* slots, double* F, double* part, int nblocks, const int* gate,
                              int want, cudaStream_t st, const int* ids, bool phys) {
    Slot* sl = reinterpret_cast<Slot*>(slots);
    SlotBO* bo = reinterpret_cast<SlotBO*>(slots + (size_t)na * cap * 8);
    cudaError_t e;
    if (ids) {
        if ((e = launch_pdl(k_rebo_geo_bo, dim3(kForceBlocks), dim3(256), 0, st, pos, hh, cnt, list, cap, sl, bo,
                            gate, want, ids)) != cudaSuccess)
            return e;
    } else {
        if ((e = launch_pdl(k_rebo_slots, dim3(kForceBlocks), dim3(256), 0, st, pos, hh, cnt, list, cap, na, sl, gate,
                            want, ids)) != cudaSuccess)
            return e;
        if ((e = launch_pdl(k_rebo_bo, dim3(kForceBlocks), dim3(256), 0, st, (const Slot*)sl, cnt, list, cap, na, bo,
                            gate, want, ids)) != cudaSuccess)
            return e;
    }
    if ((e = launch_pdl(phys ? k_rebo_force<true> : k_rebo_force<false>, dim3(nblocks), dim3(256), 0, st,
                        (const Slot*)sl, (const SlotBO*)bo, cnt, list, cap, na, F, part, gate, want, ids)) !=
        cudaSuccess)
        return e;
    return cudaGetLastError();
}

namespace {

// Occupied slots of a REBO list in atom-major order, packed into 32-lane
// bins so that no atom's slots straddle a warp: per 256-atom block one thread
// places the atoms one after another, starting a new bin when an atom's slots
// would cross one (cap <= 32), and the block's length is rounded up to whole
// bins; a scan of the block lengths then places the blocks.  Unused lanes hold
// -1.  Layout: ids[0] = padded length P, ids[1 .. P] slot ids or -1, then at
// ids[1 + 32 n + t] the partner slot of slot t.  The block size trades the
// serial placement (one thread, 256 steps) against the padding at block ends
// (at most 31 lanes per block, ~2 % of the lanes at 3 slots per atom).
constexpr int kIdsBlock = 256;

__global__ void __launch_bounds__(kIdsBlock) k_ids_count(const int* __restrict__ cnt, int cap, int n,
                                                          int* __restrict__ bsum, int* __restrict__ istart) {
    __shared__ int sm_cnt[kIdsBlock];
    const int i = blockIdx.x * kIdsBlock + threadIdx.x;
    sm_cnt[threadIdx.x] = i < n ? min(cnt[i], cap) : 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        int pos = 0;
        const int na = min(kIdsBlock, n - (int)blockIdx.x * kIdsBlock);
        for (int k = 0; k < na; k++) {
            const int m = sm_cnt[k];
            if ((pos & 31) + m > 32) pos = (pos + 31) & ~31;
            istart[blockIdx.x * kIdsBlock + k] = pos;
            pos += m;
        }
        bsum[blockIdx.x] = (pos + 31) & ~31;
    }
}

__global__ void __launch_bounds__(kIdsBlock) k_ids_emit(const int* __restrict__ cnt, int cap, int n,
                                                         const int* __restrict__ bsum,
                                                         const int* __restrict__ istart, int* __restrict__ ids) {
    __shared__ int s_base;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (w == 0) {                                  // offset of this block
        int b = 0;
        for (int k = lane; k < (int)blockIdx.x; k += 32) b += bsum[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) b += __shfl_xor_sync(kFull, b, o);
        if (lane == 0) s_base = b;
    }
    __syncthreads();
    const int base = s_base, len = bsum[blockIdx.x];
    for (int k = threadIdx.x; k < len; k += kIdsBlock) ids[1 + base + k] = -1;
    __syncthreads();
    const int i = blockIdx.x * kIdsBlock + threadIdx.x;
    if (i < n) {
        const int m = min(cnt[i], cap), off = base + istart[i];
        for (int jn = 0; jn < m; jn++) ids[1 + off + jn] = i * cap + jn;
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) ids[0] = base + len;
}

// Partner slot of every occupied slot i -> j: the position of i in j's row,
// -1 when j's row lacks i (rows cut at cap).
__global__ void k_ids_partner(const int* __restrict__ cnt, const int* __restrict__ list, int cap, int n,
                              int* __restrict__ ids) {
    const int tot = ids[0];
    int* pslot = ids + 1 + (size_t)kIdsLanes * n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += gridDim.x * blockDim.x) {
        const int t = ids[1 + k];
        if (t < 0) continue;
        const int i = t / cap;
        const int j = list[t];
        const int mj = min(cnt[j], cap);
        int pn = -1;
        for (int kn = 0; kn < mj; kn++)
            if (list[(size_t)j * cap + kn] == i) { pn = kn; break; }
        pslot[t] = pn;
    }
}

}  // namespace

int rebo_ids_scratch(int n) { return (n + kIdsBlock - 1) / kIdsBlock + n; }

cudaError_t rebo_ids_build(const int* cnt, const int* list, int cap, int n, int* ids, int* scratch, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (cap > 32) return cudaErrorInvalidValue;
    const int nb = (n + kIdsBlock - 1) / kIdsBlock;
    int* bsum = scratch;
    int* istart = scratch + nb;
    k_ids_count<<<nb, kIdsBlock, 0, st>>>(cnt, cap, n, bsum, istart);
    k_ids_emit<<<nb, kIdsBlock, 0, st>>>(cnt, cap, n, bsum, istart, ids);
    k_ids_partner<<<kForceBlocks, 256, 0, st>>>(cnt, list, cap, n, ids);
    return cudaGetLastError();
}

namespace {

// Resident blocks per SM of one LJ gather instantiation (queried once).
template <bool FV, bool F32, int U, bool PIPE, int NT>
int lj_occupancy() {
    static int occ = -1;
    if (occ < 0) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_lj_gather<FV, F32, U, PIPE, NT>, NT, 0) != cudaSuccess)
            b = 1;
        occ = b < 1 ? 1 : b;
    }
    return occ;
}

template <bool FV, bool F32, int U, bool PIPE, int NT>
int lj_dispatch(bool launch, const double* pos, const double* hh, const int* cnt, const int* list, int cap,
                const int* in_cnt, const int* in_list, int in_cap, int na, double* F, double* Facc, const LJP& p,
                double* part, cudaStream_t st, const LJPruneOut& po, int nrec, int contig) {
    const int nb = std::min(kLJMaxBlocks, lj_occupancy<FV, F32, U, PIPE, NT>() * kSMs);
    if (launch)
        launch_pdl(k_lj_gather<FV, F32, U, PIPE, NT>, dim3(nb), dim3(NT), 0, st, pos, hh, in_cnt, in_list, in_cap, na,
                   F, Facc, p, part, po, nrec, contig);
    return nb;
}

size_t staged_smem(int threads, int in_cap) {
    return (size_t)(threads / 32) * 2 * (in_cap * sizeof(int) + sizeof(uint64_t));
}

// Staged variant: grid from the occupancy at its dynamic shared memory.
template <bool FV, bool F32, int U, int NT>
int lj_dispatch_staged(bool launch, const double* pos, const double* hh, const int* in_cnt, const int* in_list,
                       int in_cap, int na, double* F, double* Facc, const LJP& p, double* part, DevErr* err,
                       cudaStream_t st, const LJPruneOut& po, int nrec, int contig) {
    static std::map<int, int> occ;                 // in_cap -> resident blocks per SM
    const size_t smem = staged_smem(NT, in_cap);
    auto it = occ.find(in_cap);
    if (it == occ.end()) {
        cudaFuncSetAttribute(k_lj_gather_staged<FV, F32, U, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
        int b = 0;
        if (smem > 200 * 1024 ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_lj_gather_staged<FV, F32, U, NT>, NT, smem) !=
                cudaSuccess)
            b = 0;
        it = occ.emplace(in_cap, b).first;
    }
    if (it->second < 1) return 0;
    const int nb = std::min(kLJMaxBlocks, it->second * kSMs);
    if (launch)
        launch_pdl(k_lj_gather_staged<FV, F32, U, NT>, dim3(nb), dim3(NT), smem, st, pos, hh, in_cnt, in_list, in_cap,
                   na, F, Facc, p, part, err, po, nrec, contig);
    return nb;
}

// Launches (launch == true) or sizes the gather of one shape; returns its grid
// (0: the shape cannot run with this row stride).
int lj_select(bool launch, int ff, int precision, const LJShape& sh, const double* pos, const double* hh,
              const int* cnt, const int* list, int cap, const int* in_cnt, const int* in_list, int in_cap, int na,
              double* F, double* Facc, double* part, cudaStream_t st, DevErr* err = nullptr,
              const LJPruneOut& po = LJPruneOut{}, int nrec = 0) {
    const LJP p = lj_params(ff);
    const bool fv = ff == FMD_FF_AIREBO, f32 = precision == FMD_PREC_FP32_PAIR;
    if (sh.pipe == 2) {
        if (in_cap % 4 != 0 || (launch && err == nullptr)) return 0;
#define FMD_LJS(FV, F32, U, NT) \
    return lj_dispatch_staged<FV, F32, U, NT>(launch, pos, hh, in_cnt, in_list, in_cap, na, F, Facc, p, part, err, st, \
                                              po, nrec, sh.contig)
#define FMD_LJS_NT(FV, F32, U) if (sh.threads == 128) { FMD_LJS(FV, F32, U, 128); } else { FMD_LJS(FV, F32, U, 256); }
#define FMD_LJS_U(FV, F32) if (sh.unroll == 2) { FMD_LJS_NT(FV, F32, 2) } else { FMD_LJS_NT(FV, F32, 4) }
        if (fv) { if (f32) { FMD_LJS_U(true, true) } else { FMD_LJS_U(true, false) } }
        else { if (f32) { FMD_LJS_U(false, true) } else { FMD_LJS_U(false, false) } }
#undef FMD_LJS_U
#undef FMD_LJS_NT
#undef FMD_LJS
    }
#define FMD_LJ_CALL(FV, F32, U, PIPE, NT) \
    return lj_dispatch<FV, F32, U, PIPE, NT>(launch, pos, hh, cnt, list, cap, in_cnt, in_list, in_cap, na, F, Facc, p, \
                                             part, st, po, nrec, sh.contig)
#define FMD_LJ_NT(FV, F32, U, PIPE) \
    if (sh.threads == 128) { FMD_LJ_CALL(FV, F32, U, PIPE, 128); } else { FMD_LJ_CALL(FV, F32, U, PIPE, 256); }
#define FMD_LJ_PIPE(FV, F32, U) if (sh.pipe) { FMD_LJ_NT(FV, F32, U, true) } else { FMD_LJ_NT(FV, F32, U, false) }
#define FMD_LJ_U(FV, F32) if (sh.unroll == 2) { FMD_LJ_PIPE(FV, F32, 2) } else { FMD_LJ_PIPE(FV, F32, 4) }
    if (fv) { if (f32) { FMD_LJ_U(true, true) } else { FMD_LJ_U(true, false) } }
    else { if (f32) { FMD_LJ_U(false, true) } else { FMD_LJ_U(false, false) } }
#undef FMD_LJ_U
#undef FMD_LJ_PIPE
#undef FMD_LJ_NT
#undef FMD_LJ_CALL
}

}  // namespace

int lj_gather_blocks(int ff, int precision, const LJShape& sh, int in_cap) {
    return lj_select(false, ff, precision, sh, nullptr, nullptr, nullptr, nullptr, 0, nullptr, nullptr, in_cap, 0,
                     nullptr, nullptr, nullptr, nullptr);
}

cudaError_t lj_gather_launch(int ff, const double* pos, const double* hh, const int* cnt, const int* list,
                             int cap, const int* in_cnt, const int* in_list, int in_cap, int na, double* F,
                             double* Facc, double* part, cudaStream_t st, int precision, const LJShape& sh,
                             DevErr* err, const LJPruneOut& po, int nrec) {
    if (lj_select(true, ff, precision, sh, pos, hh, cnt, list, cap, in_cnt, in_list, in_cap, na, F, Facc, part, st,
                  err, po, nrec) == 0)
        return cudaErrorInvalidConfiguration;
    return cudaGetLastError();
}

cudaError_t batch_lj_launch(const StepArrays* As, const int* off, int R, int nblocks, int ff, int precision,
                            int threads, int unroll, cudaStream_t st, int staged_in_cap) {
    const bool fv = ff == FMD_FF_AIREBO, f32 = precision == FMD_PREC_FP32_PAIR;
    if (staged_in_cap > 0) {
        const size_t smem = staged_smem(threads, staged_in_cap);
#define FMD_BLS(FV, F32, U, NT)                                                                               \
    {                                                                                                         \
        static bool attr = false;                                                                             \
        if (!attr) {                                                                                          \
            cudaFuncSetAttribute(k_b_lj_gather_staged<FV, F32, U, NT>,                                        \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);                    \
            attr = true;                                                                                      \
        }                                                                                                     \
        k_b_lj_gather_staged<FV, F32, U, NT><<<nblocks, NT, smem, st>>>(As, off, R, ff);                      \
    }
#define FMD_BLS_NT(FV, F32, U) if (threads == 128) FMD_BLS(FV, F32, U, 128) else FMD_BLS(FV, F32, U, 256)
#define FMD_BLS_U(FV, F32) if (unroll == 2) { FMD_BLS_NT(FV, F32, 2) } else { FMD_BLS_NT(FV, F32, 4) }
        if (fv) { if (f32) { FMD_BLS_U(true, true) } else { FMD_BLS_U(true, false) } }
        else { if (f32) { FMD_BLS_U(false, true) } else { FMD_BLS_U(false, false) } }
#undef FMD_BLS_U
#undef FMD_BLS_NT
#undef FMD_BLS
        return cudaGetLastError();
    }
#define FMD_BLJ(FV, F32, U, NT) k_b_lj_gather<FV, F32, U, NT><<<nblocks, NT, 0, st>>>(As, off, R, ff)
#define FMD_BLJ_NT(FV, F32, U) if (threads == 128) FMD_BLJ(FV, F32, U, 128); else FMD_BLJ(FV, F32, U, 256)
#define FMD_BLJ_U(FV, F32) if (unroll == 2) { FMD_BLJ_NT(FV, F32, 2); } else { FMD_BLJ_NT(FV, F32, 4); }
    if (fv) { if (f32) { FMD_BLJ_U(true, true) } else { FMD_BLJ_U(true, false) } }
    else { if (f32) { FMD_BLJ_U(false, true) } else { FMD_BLJ_U(false, false) } }
#undef FMD_BLJ_U
#undef FMD_BLJ_NT
#undef FMD_BLJ
    return cudaGetLastError();
}

cudaError_t reduce_partials(const double* part, int nblk, int nv, double* out, cudaStream_t st) {
    k_reduce<<<1, 256, 0, st>>>(part, nblk, nv, out);
    return cudaGetLastError();
}

}  // namespace fmd
