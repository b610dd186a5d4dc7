// step.cu -- NPT velocity-Verlet on the device (a17 rigid LJ:434-538,
// a18 atomistic AI:518-590 / MM:811-890) and the driver's per-step schedule
// (a19: LJ:847-897, AI:871-912, MM:1192-1236).
//
// The reference keeps xi, Vg and h on the host and synchronises several
// times per step.  Here they live in a device struct (SysScal) updated on the
// device, so a whole step -- and a list rebuild -- is
// a fixed sequence of launches with no host round trip, which is what lets
// the step be replayed as a CUDA graph:
//
//   k_begin_kick  schedule (Tt ramp, cold resets), thermostat/barostat
//               first half, scaling factors, cell update and its inverse
//               (every block on its own copy of the scalars), then the first
//               half-kick, drift in fractional coordinates, wrap, back to
//               Cartesian with the new cell (+ quaternion update)
//   forces      (airebo.cu / rigid.cu / mm.cu)
//   k_kick2_end second half-kick with per-block kinetic partials; the last
//               block to finish: force/kinetic reductions (fixed order),
//               thermostat/barostat second half, observables, rescale
//               decision, averages
//   k_rescale / k_rescale_end   cold/warm phases only
//
// Scalar arithmetic follows the reference expressions; this file is built
// with -fmad=false so they round like the reference's host code.
#include <algorithm>
#include <cmath>
#include "step.h"
#include "ljprune.h"
#include "ljprune.cuh"
#include "geom.cuh"
#include "sg_host.h"
#include "pdl.cuh"

namespace fmd {
namespace {

constexpr int kPB = 256;   // threads of per-particle kernels
constexpr int kRedThreads = 512;   // the one-block reductions of the partial records
constexpr double kMC = 12.011;

__device__ __forceinline__ double clampd(double x, double lo, double hi) {
    return x < lo ? lo : (x > hi ? hi : x);
}
__device__ __forceinline__ double inst_T(double ke, int nf) { return 2 * ke / (nf * kKB); }
__device__ __forceinline__ double inst_P(const double* W, double ke, double V) {
    return (2 * ke + W[0] + W[4] + W[8]) / (3 * V) * kEV2GPa;
}

// Thermostat + barostat half update (LJ:448-455, AI:524-530).
__device__ void npt_half(fmd_npt& s, double hdt, double ke, double ke_p, const double* W, double V,
                         double xi_lim, double vg_lim) {
    s.xi += hdt * (2 * ke - s.Nf * kKB * s.Tt) / s.Q;
    s.xi = clampd(s.xi, -xi_lim, xi_lim);
    const double dP = inst_P(W, ke_p, V) - s.Pe;
    for (int a = 0; a < 3; a++) s.Vg[a * 4] += hdt * V * dP / (s.W * kEV2GPa);
    for (int a = 0; a < 3; a++) s.Vg[a * 4] = clampd(s.Vg[a * 4], -vg_lim, vg_lim);
}

}  // namespace

__device__ void begin_body(SysScal* S, int kind, const StepParams& p) {
    fmd_npt& npt = S->npt;
    if (p.schedule) {
        const int g = ++S->gstep;
        // Tt schedule and resets (LJ:851-857)
        if (g <= p.coldstart) npt.Tt = p.T_cold;
        else if (g <= p.coldstart + p.warmup)
            npt.Tt = p.T_cold + (p.T - p.T_cold) * double(g - p.coldstart) / double(p.warmup);
        else npt.Tt = p.T;
        if (p.coldstart > 0 && g == p.coldstart + 1) {
            npt.xi = 0;
            for (int k = 0; k < 9; k++) npt.Vg[k] = 0;
        }
        if (g <= p.coldstart)
            for (int k = 0; k < 9; k++) npt.Vg[k] = 0;
    }
    const double hdt = 0.5 * p.dt;
    const bool rigid = kind == FMD_SYS_RIGID;
    if (rigid) inv9(S->h, S->hi);                                  // LJ:442
    const double V = fabs(det9(S->h));
    if (rigid) npt_half(npt, hdt, S->kt + S->kr, S->kt, S->W9, V, 0.1, 0.01);
    else npt_half(npt, hdt, S->KE, S->KE, S->W9, V, 0.05, 0.005);
    const double eps = npt.Vg[0] * S->hi[0] + npt.Vg[4] * S->hi[4] + npt.Vg[8] * S->hi[8];
    const double sc_nh = exp(-hdt * npt.xi), sc_pr = exp(-hdt * eps / 3.0);
    S->sc_nh = sc_nh;
    S->sc_v = sc_nh * sc_pr;
    for (int k = 0; k < 9; k++) S->hi_old[k] = S->hi[k];
    for (int k = 0; k < 9; k++) S->h[k] += p.dt * npt.Vg[k];          // LJ:484
    inv9(S->h, S->hi);                                                // LJ:509, AI:555
    const double eps2 = npt.Vg[0] * S->hi[0] + npt.Vg[4] * S->hi[4] + npt.Vg[8] * S->hi[8];
    S->sc_v2 = sc_nh * exp(-hdt * eps2 / 3.0);
}

namespace {

// LJ:166-174.  The reference multiplies q by the rotation increment on the
// right (q dq), which applies the lab-frame angular velocity as a body-frame
// one; left (dq q, FMD_PHYS_QUAT) rotates the lab-frame sites about the lab
// axis w, which is what the lab-frame torque update of w describes.
template <bool LEFT>
__device__ __forceinline__ void quat_step(double* q, double wx, double wy, double wz, double dt) {
    double dq[4];
    const double wm = sqrt(wx * wx + wy * wy + wz * wz), th = wm * dt * 0.5;
    if (th < 1e-14) { dq[0] = 1.0; dq[1] = 0.5 * dt * wx; dq[2] = 0.5 * dt * wy; dq[3] = 0.5 * dt * wz; }
    else { const double s = sin(th) / wm; dq[0] = cos(th); dq[1] = s * wx; dq[2] = s * wy; dq[3] = s * wz; }
    double o[4];
    if (LEFT) {
        o[0] = dq[0] * q[0] - dq[1] * q[1] - dq[2] * q[2] - dq[3] * q[3];
        o[1] = dq[0] * q[1] + dq[1] * q[0] + dq[2] * q[3] - dq[3] * q[2];
        o[2] = dq[0] * q[2] - dq[1] * q[3] + dq[2] * q[0] + dq[3] * q[1];
        o[3] = dq[0] * q[3] + dq[1] * q[2] - dq[2] * q[1] + dq[3] * q[0];
    } else {
        o[0] = q[0] * dq[0] - q[1] * dq[1] - q[2] * dq[2] - q[3] * dq[3];
        o[1] = q[0] * dq[1] + q[1] * dq[0] + q[2] * dq[3] - q[3] * dq[2];
        o[2] = q[0] * dq[2] - q[1] * dq[3] + q[2] * dq[0] + q[3] * dq[1];
        o[3] = q[0] * dq[3] + q[1] * dq[2] - q[2] * dq[1] + q[3] * dq[0];
    }
    const double nrm = sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2] + o[3] * o[3]), inv = 1.0 / nrm;
    for (int k = 0; k < 4; k++) q[k] = o[k] * inv;
}

}  // namespace

__device__ void kick_body(const StepArrays& a, double dt, int blk, int nblk, const SysScal* sc = nullptr) {
    const SysScal* S = sc ? sc : a.S;
    const double hdt = 0.5 * dt, sc_v = S->sc_v, sc_nh = S->sc_nh;
    const double* hi = S->hi_old;
    const double* h = S->h;
    const bool rigid = a.kind == FMD_SYS_RIGID;
    const double cF = rigid ? kConv / a.Mmol : kConv / kMC, cT = rigid ? kConv / a.I0 : 0.0;
    double u2 = 0.0;   // largest squared displacement since the last LJ prune
    for (int i = blk * blockDim.x + threadIdx.x; i < a.n; i += nblk * blockDim.x) {
        const double mi = (a.mass != nullptr) ? kConv / a.mass[i] : cF;
        double v[3], p[3];
        for (int c = 0; c < 3; c++) {
            v[c] = a.vel[3 * i + c] * sc_v + hdt * a.F[3 * i + c] * mi;
            a.vel[3 * i + c] = v[c];
            p[c] = a.pos[3 * i + c];
        }
        double sx = hi[0] * p[0] + hi[1] * p[1] + hi[2] * p[2];
        double sy = hi[3] * p[0] + hi[4] * p[1] + hi[5] * p[2];
        double sz = hi[6] * p[0] + hi[7] * p[1] + hi[8] * p[2];
        const double vx = hi[0] * v[0] + hi[1] * v[1] + hi[2] * v[2];
        const double vy = hi[3] * v[0] + hi[4] * v[1] + hi[5] * v[2];
        const double vz = hi[6] * v[0] + hi[7] * v[1] + hi[8] * v[2];
        sx += dt * vx; sy += dt * vy; sz += dt * vz;
        sx -= floor(sx); sy -= floor(sy); sz -= floor(sz);
        a.pos[3 * i] = h[0] * sx + h[1] * sy + h[2] * sz;
        a.pos[3 * i + 1] = h[3] * sx + h[4] * sy + h[5] * sz;
        a.pos[3 * i + 2] = h[6] * sx + h[7] * sy + h[8] * sz;
        if (a.prune_sb) {
            // nearest-image fractional displacement, measured in the new cell
            double ex = sx - a.prune_sb[3 * i], ey = sy - a.prune_sb[3 * i + 1], ez = sz - a.prune_sb[3 * i + 2];
            ex -= rint(ex); ey -= rint(ey); ez -= rint(ez);
            const double ux = h[0] * ex + h[1] * ey + h[2] * ez, uy = h[3] * ex + h[4] * ey + h[5] * ez,
                         uz = h[6] * ex + h[7] * ey + h[8] * ez;
            u2 = fmax(u2, ux * ux + uy * uy + uz * uz);
        }
        if (rigid) {
            double w[3];
            for (int c = 0; c < 3; c++) {
                w[c] = a.omg[3 * i + c] * sc_nh + hdt * a.T[3 * i + c] * cT;
                a.omg[3 * i + c] = w[c];
            }
            if (a.quat_left) quat_step<true>(a.qv + 4 * i, w[0], w[1], w[2], dt);
            else quat_step<false>(a.qv + 4 * i, w[0], w[1], w[2], dt);     // LJ:503-508
        }
    }
    if (a.prune_sb) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) u2 = fmax(u2, __shfl_xor_sync(kFull, u2, o));
        if ((threadIdx.x & 31) == 0 && u2 > 0.0)
            atomicMax(a.prune_umax, (unsigned long long)__double_as_longlong(sqrt(u2) * (1.0 + 1e-12)));
    }
}

// Second half-kick with per-block sums of m v^2 (atomistic) or v^2 and w^2
// (rigid) into part_ke[2 * blk]; sm holds 64 doubles.
__device__ void kick2_body(const StepArrays& a, double dt, int blk, int nblk, double* sm) {
    const SysScal* S = a.S;
    const double hdt = 0.5 * dt, sc_v2 = S->sc_v2, sc_nh = S->sc_nh;
    const bool rigid = a.kind == FMD_SYS_RIGID;
    const double cF = rigid ? kConv / a.Mmol : kConv / kMC, cT = rigid ? kConv / a.I0 : 0.0;
    double acc[2] = {0.0, 0.0};
    for (int i = blk * blockDim.x + threadIdx.x; i < a.n; i += nblk * blockDim.x) {
        const double mi = (a.mass != nullptr) ? kConv / a.mass[i] : cF;
        double vv = 0;
        for (int c = 0; c < 3; c++) {
            const double v = (a.vel[3 * i + c] + hdt * a.F[3 * i + c] * mi) * sc_v2;
            a.vel[3 * i + c] = v;
            vv += v * v;
        }
        if (rigid) {
            double ww = 0;
            for (int c = 0; c < 3; c++) {
                const double w = (a.omg[3 * i + c] + hdt * a.T[3 * i + c] * cT) * sc_nh;
                a.omg[3 * i + c] = w;
                ww += w * w;
            }
            acc[0] += vv;
            acc[1] += ww;
        } else {
            acc[0] += (a.mass != nullptr ? a.mass[i] : kMC) * vv;
        }
    }
    block_sum_store<2>(acc, sm, a.part_ke + 2 * blk);
}

namespace {

// The start of a step and the first half-kick with drift in one launch: every
// block copies the step scalars into shared memory and runs the thermostat,
// barostat and cell update on its copy (the same arithmetic on the same
// inputs, so every copy is the same), kicks and drifts its particles with
// them and takes a ticket; the last block, once every block has read the old
// scalars, writes its copy back and so resets the ticket.
__global__ void __launch_bounds__(kPB) k_begin_kick(StepArrays a, StepParams p) {
    FMD_PDL_WAIT();
    __shared__ SysScal sS;
    __shared__ bool last;
    static_assert(sizeof(SysScal) % sizeof(int) == 0, "SysScal copied as words");
    constexpr int kWords = sizeof(SysScal) / sizeof(int);
    const int* src = reinterpret_cast<const int*>(a.S);
    int* dst = reinterpret_cast<int*>(&sS);
    for (int k = threadIdx.x; k < kWords; k += blockDim.x) dst[k] = src[k];
    __syncthreads();
    if (threadIdx.x == 0) begin_body(&sS, a.kind, p);
    __syncthreads();
    kick_body(a, p.dt, blockIdx.x, gridDim.x, &sS);
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&a.S->kick_done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    int* out = reinterpret_cast<int*>(a.S);
    for (int k = threadIdx.x; k < kWords; k += blockDim.x) out[k] = dst[k];   // kick_done: 0 again
}

__global__ void __launch_bounds__(kPB) k_ke_partial(StepArrays a) {
    __shared__ double sm[32 * 2];
    const bool rigid = a.kind == FMD_SYS_RIGID;
    double acc[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const double vv = a.vel[3 * i] * a.vel[3 * i] + a.vel[3 * i + 1] * a.vel[3 * i + 1] +
                          a.vel[3 * i + 2] * a.vel[3 * i + 2];
        if (rigid) {
            acc[0] += vv;
            acc[1] += a.omg[3 * i] * a.omg[3 * i] + a.omg[3 * i + 1] * a.omg[3 * i + 1] +
                      a.omg[3 * i + 2] * a.omg[3 * i + 2];
        } else {
            acc[0] += (a.mass != nullptr ? a.mass[i] : kMC) * vv;
        }
    }
    block_sum_store<2>(acc, sm, a.part_ke + 2 * blockIdx.x);
}

}  // namespace

__device__ void rescale_body(const StepArrays& a, int blk, int nblk, double* sm) {
    const SysScal* S = a.S;
    const bool rigid = a.kind == FMD_SYS_RIGID;
    const bool doit = S->do_rescale != 0;
    const double sc = S->scale;
    double acc[2] = {0.0, 0.0};
    for (int i = blk * blockDim.x + threadIdx.x; i < a.n; i += nblk * blockDim.x) {
        double vv = 0, ww = 0;
        for (int c = 0; c < 3; c++) {
            double v = a.vel[3 * i + c];
            if (doit) { v *= sc; a.vel[3 * i + c] = v; }
            vv += v * v;
            if (rigid) {
                double w = a.omg[3 * i + c];
                if (doit) { w *= sc; a.omg[3 * i + c] = w; }
                ww += w * w;
            }
        }
        if (rigid) { acc[0] += vv; acc[1] += ww; }
        else acc[0] += (a.mass != nullptr ? a.mass[i] : kMC) * vv;
    }
    block_sum_store<2>(acc, sm, a.part_ke + 2 * blk);
}

namespace {

__global__ void __launch_bounds__(kPB) k_rescale(StepArrays a) {
    FMD_PDL_WAIT();
    __shared__ double sm[32 * 2];
    rescale_body(a, blockIdx.x, gridDim.x, sm);
}

// One pass over every partial array: each thread sums its strided records
// (fixed order), then one CTA reduction for all fields.  Layout of t[]:
// [0,10) part_f1 fields, [10,20) part_f2 fields, [20] part_f3, [21,23) kinetic.
constexpr int kRedFields = 23;

__device__ void reduce_all(const StepArrays& a, int nblk_f1, int nblk_ke, bool forces, bool kinetic,
                           double* sm, double (&t)[kRedFields], int nblk_f2) {
    double acc[kRedFields];
#pragma unroll
    for (int k = 0; k < kRedFields; k++) acc[k] = 0.0;
    // L2 loads (__ldcg): the fused second kick reduces records that other
    // blocks of the same launch have just written.
    if (forces) {
        // record widths as compile-time constants so each thread's loads issue together
        if (a.kind == FMD_SYS_MM) {
            for (int b = threadIdx.x; b < nblk_f1; b += blockDim.x)
#pragma unroll
                for (int k = 0; k < kMMNV; k++) acc[k] += __ldcg(a.part_f1 + (size_t)b * kMMNV + k);
        } else {
            for (int b = threadIdx.x; b < nblk_f1; b += blockDim.x)
#pragma unroll
                for (int k = 0; k < kNV; k++) acc[k] += __ldcg(a.part_f1 + (size_t)b * kNV + k);
        }
        if (a.kind != FMD_SYS_RIGID)
            for (int b = threadIdx.x; b < nblk_f2; b += blockDim.x) {
#pragma unroll
                for (int k = 0; k < kNV; k++) acc[10 + k] += __ldcg(a.part_f2 + (size_t)b * kNV + k);
            }
        if (a.kind == FMD_SYS_MM && a.has_charge)
            for (int b = threadIdx.x; b < kForceBlocks; b += blockDim.x) acc[20] += __ldcg(a.part_f3 + b);
        // the switched-LJ correction belongs to the LJ term
        if (a.kind == FMD_SYS_AIREBO && (a.rebo2_flags & FMD_REBO2_LJ_SWITCH))
            for (int b = threadIdx.x; b < kForceBlocks; b += blockDim.x) {
#pragma unroll
                for (int k = 0; k < kNV; k++) acc[10 + k] += __ldcg(a.part_sw + (size_t)b * kNV + k);
            }
    }
    if (kinetic)
        for (int b = threadIdx.x; b < nblk_ke; b += blockDim.x) {
            acc[21] += __ldcg(a.part_ke + 2 * b);
            acc[22] += __ldcg(a.part_ke + 2 * b + 1);
        }
    block_sum_store<kRedFields>(acc, sm, t);   // result valid in thread 0
}

// Thread 0: kinetic energies from the reduced sums into S (a.S or a copy).
__device__ void kinetic_from_sums(SysScal* S, const StepArrays& a, const double (&t)[kRedFields]) {
    if (a.kind == FMD_SYS_RIGID) {
        S->kt = 0.5 * a.Mmol * t[21] / kConv;     // LJ:411
        S->kr = 0.5 * a.I0 * t[22] / kConv;       // LJ:420
        S->KE = S->kt + S->kr;
    } else {
        S->KE = 0.5 * t[21] / kConv;              // AI:506, MM:799
    }
}

// Thread 0: virial and energies (program grouping) from the reduced sums
// into S (a.S or a copy).
__device__ void forces_from_sums(SysScal* S, const StepArrays& a, const double (&t)[kRedFields]) {
    double e[8] = {0, 0, 0, 0, 0, 0, 0, 0}, w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (a.kind == FMD_SYS_RIGID) {
        e[0] = t[0];
        for (int q = 0; q < 9; q++) w[q] = t[1 + q];
    } else if (a.kind == FMD_SYS_AIREBO) {
        e[1] = t[0]; e[2] = t[10]; e[0] = e[1] + e[2];
        for (int q = 0; q < 9; q++) w[q] = t[1 + q] + t[11 + q];
    } else {
        for (int q = 0; q < 4; q++) e[q] = t[q];
        e[4] = t[10];
        e[5] = a.has_charge ? t[20] : 0.0;
        e[6] = e[0] + e[1] + e[2] + e[3] + e[4] + e[5];
        const int d[3] = {0, 4, 8};
        for (int q = 0; q < 3; q++) w[d[q]] = t[4 + q] + t[11 + d[q]];
    }
    for (int q = 0; q < 9; q++) S->W9[q] = w[q];
    for (int q = 0; q < 8; q++) S->E[q] = e[q];
}

// Observables, averages and the monitor record (LJ:874-897, AI:896-912, MM:1215-1236).
__device__ void record(SysScal* S, int kind, const StepParams& p) {
    const int g = S->gstep;
    const double an = S->h[0] / p.nc;
    S->an = an;
    if (g >= p.gavg_from && g <= p.gavg_to) {
        fmd_avg& A = S->avg;
        A.sT += S->Tn; A.sP += S->Pn; A.sa += an;
        if (kind == FMD_SYS_RIGID) {
            A.sE[0] += S->E[0] / p.nmol;
        } else if (kind == FMD_SYS_AIREBO) {
            A.sE[0] += S->E[1] / p.nmol; A.sE[1] += S->E[2] / p.nmol; A.sE[2] += S->E[0] / p.nmol;
        } else {
            A.sE[0] += S->E[0] / p.nmol; A.sE[1] += S->E[1] / p.nmol;
            A.sE[2] += (S->E[2] + S->E[3]) / p.nmol; A.sE[3] += S->E[4] / p.nmol;
            A.sE[4] += S->E[6] / p.nmol;
        }
        A.n++;
    }
    fmd_obs& o = S->obs;
    o.step = g; o.T = S->Tn; o.P = S->Pn; o.a = an; o.KE = S->KE;
    for (int q = 0; q < 8; q++) o.E[q] = S->E[q];
}

}  // namespace

// After the LJ gather of a force evaluation (thread 0 of its reduction): when
// that gather pruned (the same decision on the same inputs), the displacement
// bound restarts from this step's positions and cell hh; counts evaluations
// and prunes.
__device__ void lj_prune_commit(const StepArrays& a, const double* hh) {
    if (!a.prune_hb || !(a.prune_delta > 0.0)) return;
    if (lj_prune_needed(a.prune_umax, hh, a.prune_hb, a.prune_delta, a.prune_rc)) {
        *a.prune_umax = 0ull;
        for (int q = 0; q < 9; q++) a.prune_hb[q] = hh[q];
        a.prune_stats[1] += 1ull;
    }
    a.prune_stats[0] += 1ull;
}

// Thread 0 of the step end: prune commit, energies, virial and kinetic
// energy from the reduced sums, the thermostat/barostat second half and the
// driver's observables, on the scalars S.
__device__ void end_scalars(const StepArrays& a, const StepParams& p, const double (&t)[kRedFields], SysScal* S) {
    lj_prune_commit(a, S->h);
    forces_from_sums(S, a, t);
    kinetic_from_sums(S, a, t);
    const double hdt = 0.5 * p.dt;
    const bool rigid = a.kind == FMD_SYS_RIGID;
    const double V2 = fabs(det9(S->h));
    if (rigid) npt_half(S->npt, hdt, S->KE, S->kt, S->W9, V2, 0.1, 0.01);
    else npt_half(S->npt, hdt, S->KE, S->KE, S->W9, V2, 0.05, 0.005);
    if (!p.schedule) return;
    // Driver observables after step_npt (LJ:874-876, AI:896, MM:1215-1219).
    const double V = fabs(det9(S->h));
    S->Tn = inst_T(S->KE, S->npt.Nf);
    S->Pn = inst_P(S->W9, rigid ? S->kt : S->KE, V);
    const int g = S->gstep;
    const bool phase = (g <= p.coldstart || g <= p.coldstart + p.warmup);
    S->do_rescale = 0;
    if (phase && S->Tn > 0.1) {                                      // LJ:879-894
        const double tgt = (g <= p.coldstart) ? p.T_cold : S->npt.Tt;
        S->scale = sqrt(fmax(tgt, 0.1) / S->Tn);
        S->do_rescale = 1;
    }
    if (!phase) record(S, a.kind, p);
}

// The end of a step in one block: the block copies the step scalars into
// shared memory (sS) and reduces the partial records, thread 0 runs the
// scalar end on that copy (shared-memory latency on its serial chain instead
// of global), and the block writes the copy back with the block ticket
// kick2_done reset.  No other block reads the scalars meanwhile.
__device__ void end_body(const StepArrays& a, const StepParams& p, int nblk_f1, int nblk_ke, int nblk_f2,
                         double* sm, SysScal* sS) {
    static_assert(sizeof(SysScal) % sizeof(int) == 0, "SysScal copied as words");
    constexpr int kWords = sizeof(SysScal) / sizeof(int);
    int* gS = reinterpret_cast<int*>(a.S);
    int* cS = reinterpret_cast<int*>(sS);
    for (int k = threadIdx.x; k < kWords; k += blockDim.x) cS[k] = __ldcg(gS + k);
    __syncthreads();
    double t[kRedFields];
    reduce_all(a, nblk_f1, nblk_ke, true, true, sm, t, nblk_f2);
    if (threadIdx.x == 0) {
        end_scalars(a, p, t, sS);
        sS->kick2_done = 0u;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kWords; k += blockDim.x) gS[k] = cS[k];
}

__device__ void rescale_end_body(const StepArrays& a, const StepParams& p, int nblk_ke, double* sm) {
    SysScal* S = a.S;
    const bool doit = S->do_rescale != 0;
    double t[kRedFields];
    if (doit) reduce_all(a, 0, nblk_ke, false, true, sm, t, 0);
    if (threadIdx.x != 0) return;
    if (doit) {
        kinetic_from_sums(S, a, t);
        S->Tn = inst_T(S->KE, S->npt.Nf);
        S->npt.xi = 0;
        if (S->gstep <= p.coldstart)
            for (int k = 0; k < 9; k++) S->npt.Vg[k] = 0;
    }
    record(S, a.kind, p);
}

namespace {

// The second half-kick and the end of the step in one launch: every block
// writes its kinetic partial and takes a ticket; the last block to finish
// runs end_body (the same fixed-order reduction of all partial records, so
// the result does not depend on which block is last) and resets the ticket.
__global__ void __launch_bounds__(kPB) k_kick2_end(StepArrays a, StepParams p, int nblk_f1) {
    FMD_PDL_WAIT();
    __shared__ double sm[32 * kRedFields];
    __shared__ SysScal sS;
    __shared__ bool last;
    kick2_body(a, p.dt, blockIdx.x, gridDim.x, sm);
    __threadfence();                      // this block's partial before its ticket
    if (threadIdx.x == 0) last = atomicAdd(&a.S->kick2_done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    end_body(a, p, nblk_f1, gridDim.x, a.lj_blocks, sm, &sS);   // resets kick2_done
}

__global__ void __launch_bounds__(kRedThreads) k_rescale_end(StepArrays a, StepParams p, int nblk_ke) {
    FMD_PDL_WAIT();
    __shared__ double sm[32 * kRedFields];
    rescale_end_body(a, p, nblk_ke, sm);
}

__global__ void __launch_bounds__(kRedThreads) k_ke_final(StepArrays a, int nblk_ke) {
    __shared__ double sm[32 * kRedFields];
    double t[kRedFields];
    reduce_all(a, 0, nblk_ke, false, true, sm, t, 0);
    if (threadIdx.x == 0) kinetic_from_sums(a.S, a, t);
}

// ---- replica batch: each single-system kernel once over all replicas ----
__global__ void k_b_begin(BatchDev b) {
    if (threadIdx.x != 0) return;
    const StepArrays& a = b.A[blockIdx.x];
    begin_body(a.S, a.kind, b.P[blockIdx.x]);
}

__global__ void __launch_bounds__(kPB) k_b_kick(BatchDev b) {
    const int r = batch_rep(b.off_atom, b.R, blockIdx.x);
    kick_body(b.A[r], b.P[r].dt, blockIdx.x - b.off_atom[r], b.off_atom[r + 1] - b.off_atom[r]);
}

__global__ void __launch_bounds__(kPB) k_b_kick2(BatchDev b) {
    __shared__ double sm[32 * 2];
    const int r = batch_rep(b.off_atom, b.R, blockIdx.x);
    kick2_body(b.A[r], b.P[r].dt, blockIdx.x - b.off_atom[r], b.off_atom[r + 1] - b.off_atom[r], sm);
}

__global__ void __launch_bounds__(kPB) k_b_rescale(BatchDev b) {
    __shared__ double sm[32 * 2];
    const int r = batch_rep(b.off_atom, b.R, blockIdx.x);
    rescale_body(b.A[r], blockIdx.x - b.off_atom[r], b.off_atom[r + 1] - b.off_atom[r], sm);
}

__global__ void __launch_bounds__(256) k_b_end(BatchDev b) {
    __shared__ double sm[32 * kRedFields];
    __shared__ SysScal sS;
    const int r = blockIdx.x;
    end_body(b.A[r], b.P[r], b.off_f1[r + 1] - b.off_f1[r], b.off_atom[r + 1] - b.off_atom[r],
             b.off_lj[r + 1] - b.off_lj[r], sm, &sS);
}

__global__ void __launch_bounds__(256) k_b_rescale_end(BatchDev b) {
    __shared__ double sm[32 * kRedFields];
    const int r = blockIdx.x;
    rescale_end_body(b.A[r], b.P[r], b.off_atom[r + 1] - b.off_atom[r], sm);
}

__global__ void __launch_bounds__(kRedThreads) k_force_final(StepArrays a, int nblk_f1) {
    __shared__ double sm[32 * kRedFields];
    double t[kRedFields];
    reduce_all(a, nblk_f1, 0, true, false, sm, t, a.lj_blocks);
    if (threadIdx.x == 0) {
        forces_from_sums(a.S, a, t);
        lj_prune_commit(a, a.S->h);
    }
}

}  // namespace

int force_partial_blocks(const StepArrays& a) {
    return a.kind == FMD_SYS_RIGID ? rigid_grid(a.n) : (a.kind == FMD_SYS_AIREBO ? a.rebo_blocks : kForceBlocks);
}

// LJ term of an atomistic system: the gather over the full rows, or with
// pruned rows the gather that decides per evaluation between pruning the full
// rows and walking the pruned ones.
cudaError_t enqueue_lj(const StepArrays& a, int ff, cudaStream_t st) {
    const double* hh = a.S->h;
    if (!a.prune || a.prune->delta <= 0.0)
        return lj_gather_launch(ff, a.pos, hh, a.cnt_a, a.list_a, a.cap_a, a.in_cnt, a.in_list, a.in_cap, a.n, a.F,
                                a.Facc, a.part_f2, st, a.precision, a.lj_shape, a.err, LJPruneOut{}, a.lj_blocks);
    // one launch: each block decides whether this evaluation prunes (full
    // rows, pruned rows written) or walks the pruned rows; the step's
    // reduction then restarts the displacement bound (lj_prune_commit)
    return lj_gather_launch(ff, a.pos, hh, a.cnt_a, a.list_a, a.cap_a, a.in_cnt, a.in_list, a.in_cap, a.n, a.F,
                            a.Facc, a.part_f2, st, a.precision, a.lj_shape_p, a.err, lj_prune_out(*a.prune),
                            a.lj_blocks);
}

cudaError_t enqueue_forces(const StepArrays& a, cudaStream_t st, bool judge) {
    cudaError_t e = cudaSuccess;
    const double* hh = a.S->h;
    if (a.kind == FMD_SYS_RIGID) {
        e = rigid_launch(a.precision, a.pos, a.qv, a.body, hh, a.cnt_a, a.list_a, a.cap_a, a.n, a.natom,
                         a.rmcut2, a.F, a.T, a.part_f1, st, a.rigid_lab, a.rigid_shape);
    } else if (a.kind == FMD_SYS_AIREBO) {
        if (a.rebo2_flags & FMD_REBO2_BOND_ORDER)
            e = rebo2_launch(a.rebo2, a.pos, hh, a.cnt_b, a.list_b, a.cap_b, a.n, a.Facc, a.part_f1, a.rebo_blocks,
                             st);
        else if (a.sg) e = sg_enqueue_rebo(*a.sg, a, judge, st);
        else if (a.rebo_slots)
            e = rebo_slots_launch(a.pos, hh, a.cnt_b, a.list_b, a.cap_b, a.n, a.rebo_slots, a.Facc, a.part_f1,
                                  kForceBlocks, nullptr, 0, st, a.rebo_ids, a.rebo_phys != 0);
        else e = rebo_launch(a.pos, hh, a.cnt_b, a.list_b, a.cap_b, a.n, a.Facc, a.part_f1, st);
        if (e != cudaSuccess) return e;
        e = enqueue_lj(a, FMD_FF_AIREBO, st);
        // the switched LJ: its correction adds into the finished F
        if (e == cudaSuccess && (a.rebo2_flags & FMD_REBO2_LJ_SWITCH))
            e = lj_switch_launch(a.rebo2, a.pos, hh, a.cnt_b, a.list_b, a.cap_b, a.cnt_a, a.list_a, a.cap_a, a.n,
                                 a.F, a.part_sw, kForceBlocks, (a.rebo2_flags & FMD_REBO2_BOND_ORDER) != 0, st);
    } else {
        if ((e = mm_bonded_launch(a.topo, a.pos, hh, a.Facc, a.part_f1, st)) != cudaSuccess) return e;
        if (a.has_charge)
            if ((e = mm_coulomb_launch(a.pos, hh, a.charge, a.mol_id, a.n, a.Facc, a.part_f3, st)) != cudaSuccess) return e;
        e = enqueue_lj(a, FMD_FF_MM, st);
    }
    return e;
}

cudaError_t enqueue_force_reduce(const StepArrays& a, cudaStream_t st) {
    k_force_final<<<1, kRedThreads, 0, st>>>(a, force_partial_blocks(a));
    return cudaGetLastError();
}

cudaError_t enqueue_ke(const StepArrays& a, cudaStream_t st) {
    k_ke_partial<<<kForceBlocks, kPB, 0, st>>>(a);
    k_ke_final<<<1, kRedThreads, 0, st>>>(a, kForceBlocks);
    return cudaGetLastError();
}

cudaError_t enqueue_step(const StepArrays& a, const StepParams& p, bool rescale_phase, cudaStream_t st,
                         bool judge) {
    cudaError_t e;
    // programmatic dependent launches: each kernel's launch overlaps the
    // previous one's tail (pdl.cuh)
    // per-particle kernels: one thread per particle (grid-stride beyond kForceBlocks)
    const int pblocks = std::max(1, std::min(kForceBlocks, (a.n + kPB - 1) / kPB));
    if ((e = launch_pdl(k_begin_kick, dim3(pblocks), dim3(kPB), 0, st, a, p)) != cudaSuccess) return e;
    if ((e = enqueue_forces(a, st, judge)) != cudaSuccess) return e;
    if ((e = launch_pdl(k_kick2_end, dim3(pblocks), dim3(kPB), 0, st, a, p, force_partial_blocks(a))) != cudaSuccess)
        return e;
    if (rescale_phase && p.schedule) {
        if ((e = launch_pdl(k_rescale, dim3(kForceBlocks), dim3(kPB), 0, st, a)) != cudaSuccess) return e;
        if ((e = launch_pdl(k_rescale_end, dim3(1), dim3(kRedThreads), 0, st, a, p, kForceBlocks)) != cudaSuccess)
            return e;
    }
    return cudaGetLastError();
}

cudaError_t enqueue_batch_step(const BatchDev& b, bool rescale_phase, cudaStream_t st) {
    cudaError_t e;
    k_b_begin<<<b.R, 32, 0, st>>>(b);
    k_b_kick<<<b.nblk_atom, kPB, 0, st>>>(b);
    if (b.kind == FMD_SYS_MM)
        if ((e = batch_mm_bonded_launch(b.A, b.off_f1, b.R, b.nblk_f1, b.f1_threads, st)) != cudaSuccess) return e;
    if ((e = batch_lj_launch(b.A, b.off_lj, b.R, b.nblk_lj, b.ff, b.precision, b.lj_threads, b.lj_unroll, st,
                             b.lj_staged_in_cap)) != cudaSuccess)
        return e;
    k_b_kick2<<<b.nblk_atom, kPB, 0, st>>>(b);
    k_b_end<<<b.R, 256, 0, st>>>(b);
    if (rescale_phase) {
        k_b_rescale<<<b.nblk_atom, kPB, 0, st>>>(b);
        k_b_rescale_end<<<b.R, 256, 0, st>>>(b);
    }
    return cudaGetLastError();
}

}  // namespace fmd
