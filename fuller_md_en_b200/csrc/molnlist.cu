// molnlist.cu -- neighbour lists of atomistic systems whose molecules are
// contiguous index ranges (every crystal the reference builds: AI:781-786,
// MM:1094-1111), bit-exact with the reference's O(N^2) builders
// (build_nlist_rebo AI:251-261, build_nlist_lj AI:263-272, MM:337-346).
//
// With contiguous molecules, j > i between different molecules means
// molecule(j) > molecule(i), so the half-list row of atom i is the accepted
// atoms of the higher-numbered neighbour molecules in ascending order: the row
// comes out sorted without a bitmap, its first `cap` entries are the
// reference's truncation, and the candidates of one molecule are contiguous
// in memory (coalesced loads).  The LJ gather's full rows (incoming entries,
// then the row) come from the walk's candidate bitmap when every molecule has
// 32-64 atoms (k_mol_incoming), else from the transpose of the half rows
// (nlist_transpose, nlist.cu), as they do after a cell-grid build.
// Intramolecular (REBO) rows walk the atom's own molecule.
//
// Candidate molecules: a centre c and radius R per molecule, and molecule
// pairs with |c_A - c_B| <= rc + R_A + R_B (minimum image).  For a diagonal
// cell the reference's minimum image is the true nearest image per axis, the
// distance is a metric on the torus, and the triangle inequality makes the
// molecule test conservative.  For other cells, when a molecule has more
// partners than the table holds (a disintegrating crystal), the system falls
// back to the cell-grid builder (nlist.cu) for that rebuild: a device flag
// gates the two paths inside one CUDA graph.
#include <cmath>

#include "geom.cuh"
#include "kernels.h"
#include "ljprune.h"
#include "molnlist.h"

namespace fmd {
namespace {

constexpr double kScreenMax = 2048.0;   // coordinate and cell-edge bound of the FP32 screen (A)

__device__ __forceinline__ bool diag_cell(const double* h, const double* hi) {
    return h[1] == 0.0 && h[2] == 0.0 && h[3] == 0.0 && h[5] == 0.0 && h[6] == 0.0 && h[7] == 0.0 &&
           hi[1] == 0.0 && hi[2] == 0.0 && hi[3] == 0.0 && hi[5] == 0.0 && hi[6] == 0.0 && hi[7] == 0.0;
}

// One component of the reference's minimum image in a diagonal cell (the
// general formula with zero off-diagonals; round(s) by comparisons for |s| < 1.5).
__device__ __forceinline__ double mimg_axis(double d, double hii, double hii_inv) {
    double s = __dmul_rn(hii_inv, d);
    double r = s >= 0.5 ? 1.0 : (s <= -0.5 ? -1.0 : 0.0);
    if (!(fabs(s) < 1.5)) r = round(s);
    s = __dsub_rn(s, r);
    return __dmul_rn(hii, s);
}

// The reference's pair test r^2 < rc2 for d = pos[j] - pos[i] (AI:258, 268).
__device__ __forceinline__ bool pair_in(const double* __restrict__ pos, int i, int j, const double* h,
                                        const double* hi, bool diag, double rc2) {
    double dx = __dsub_rn(pos[3 * j], pos[3 * i]), dy = __dsub_rn(pos[3 * j + 1], pos[3 * i + 1]),
           dz = __dsub_rn(pos[3 * j + 2], pos[3 * i + 2]);
    if (diag) {
        dx = mimg_axis(dx, h[0], hi[0]);
        dy = mimg_axis(dy, h[4], hi[4]);
        dz = mimg_axis(dz, h[8], hi[8]);
    } else {
        mimg(dx, dy, dz, hi, h);
    }
    return norm2_rn(dx, dy, dz) < rc2;
}

// Centre (mean of the minimum images relative to the first atom) and radius
// (largest minimum-image distance of an atom from the centre) per molecule,
// and the FP32 copy of the positions; one warp per molecule.  Resets the
// partner-overflow flag.
__device__ __forceinline__ void mol_centre_body(const double* __restrict__ pos, const double* __restrict__ hh,
                                                const int* __restrict__ off, int M, double* __restrict__ cen,
                                                double* __restrict__ rad, float4* __restrict__ pos32,
                                                int* __restrict__ flag, int blk) {
    const double* h = hh;
    const double* hi = hh + 9;
    const int lane = threadIdx.x & 31;
    const int w = (blk * blockDim.x + threadIdx.x) >> 5;
    if (blk == 0 && threadIdx.x == 0) flag[1] = 0;
    if (w >= M) return;
    const int a0 = off[w], a1 = off[w + 1];
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int a = a0 + lane; a < a1; a += 32) {
        double dx = pos[3 * a] - pos[3 * a0], dy = pos[3 * a + 1] - pos[3 * a0 + 1], dz = pos[3 * a + 2] - pos[3 * a0 + 2];
        const double x = pos[3 * a], y = pos[3 * a + 1], z = pos[3 * a + 2];
        const bool small = fabs(x) < kScreenMax && fabs(y) < kScreenMax && fabs(z) < kScreenMax;
        pos32[a] = make_float4((float)x, (float)y, (float)z, small ? 1.0f : 0.0f);
        mimg(dx, dy, dz, hi, h);
        sx += dx; sy += dy; sz += dz;
    }
    sx = warp_sum(sx); sy = warp_sum(sy); sz = warp_sum(sz);
    const double inv = 1.0 / (a1 - a0);
    const double cx = pos[3 * a0] + sx * inv, cy = pos[3 * a0 + 1] + sy * inv, cz = pos[3 * a0 + 2] + sz * inv;
    double r2 = 0.0;
    for (int a = a0 + lane; a < a1; a += 32) {
        double dx = pos[3 * a] - cx, dy = pos[3 * a + 1] - cy, dz = pos[3 * a + 2] - cz;
        mimg(dx, dy, dz, hi, h);
        r2 = fmax(r2, dx * dx + dy * dy + dz * dz);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r2 = fmax(r2, __shfl_xor_sync(kFull, r2, o));
    if (lane == 0) {
        cen[3 * w] = cx; cen[3 * w + 1] = cy; cen[3 * w + 2] = cz;
        rad[w] = sqrt(r2);
    }
}

__global__ void k_mol_centre(const double* __restrict__ pos, const double* __restrict__ hh,
                             const int* __restrict__ off, int M, double* __restrict__ cen, double* __restrict__ rad,
                             float4* __restrict__ pos32, int* __restrict__ flag) {
    mol_centre_body(pos, hh, off, M, cen, rad, pos32, flag, blockIdx.x);
}

// Partner molecules of each molecule (both directions, ascending); one warp
// per molecule.  flag[0] = 1 when the molecule path is valid for this
// rebuild (diagonal cell, no table overflow), else 0.
__device__ __forceinline__ void mol_pairs_body(const double* __restrict__ hh, int M, const double* __restrict__ cen,
                                               const double* __restrict__ rad, double rc, int pmax,
                                               int* __restrict__ npart, int* __restrict__ part,
                                               int* __restrict__ flag, int blk) {
    const double* h = hh;
    const double* hi = hh + 9;
    const int lane = threadIdx.x & 31;
    const int A = (blk * blockDim.x + threadIdx.x) >> 5;
    if (A >= M) return;
    const double cx = cen[3 * A], cy = cen[3 * A + 1], cz = cen[3 * A + 2], ra = rad[A];
    int n = 0;
    for (int b0 = 0; b0 < M; b0 += 32) {
        const int B = b0 + lane;
        bool ok = false;
        if (B < M && B != A) {
            double dx = cen[3 * B] - cx, dy = cen[3 * B + 1] - cy, dz = cen[3 * B + 2] - cz;
            mimg(dx, dy, dz, hi, h);
            const double lim = (rc + (ra + rad[B])) * (1.0 + 1e-9) + 1e-6;   // rounding margin; symmetric in A, B
            ok = dx * dx + dy * dy + dz * dz <= lim * lim;
        }
        const unsigned m = __ballot_sync(kFull, ok);
        const int k = n + __popc(m & ((1u << lane) - 1u));
        if (ok && k < pmax) part[(size_t)A * pmax + k] = B;
        n += __popc(m);
    }
    if (lane == 0) {
        npart[A] = n < pmax ? n : pmax;
        if (n > pmax) atomicOr(&flag[1], 1);
    }
}

__global__ void k_mol_pairs(const double* __restrict__ hh, int M, const double* __restrict__ cen,
                            const double* __restrict__ rad, double rc, int pmax, int* __restrict__ npart,
                            int* __restrict__ part, int* __restrict__ flag) {
    mol_pairs_body(hh, M, cen, rad, rc, pmax, npart, part, flag, blockIdx.x);
}

__global__ void k_mol_decide(const double* __restrict__ hh, int* __restrict__ flag) {
    if (threadIdx.x == 0) flag[0] = (diag_cell(hh, hh + 9) && flag[1] == 0) ? 1 : 0;
}

// FP32 screen of the reference's test r^2 < rc2 (diagonal cell): positions
// rounded to FP32 (error <= 2^-24 * 2048 = 1.2e-4 A per coordinate when
// |x| < kScreenMax; <= 4e-6 A below 128 A), difference and nearest image in
// FP32 (rintf, as the FP64 image for |d| well below half the cell), so r^2 at
// r ~ 12 A is off by less than 0.016 A^2 (1e-3 A^2 below 128 A).  Outside a
// band of +-kScreenBand around rc2 its verdict is the FP64 one; inside, the
// FP64 test decides.  Used when half the narrowest cell edge exceeds the list
// radius by 1 A (no candidate near the radius sits near a half-cell image
// switch), every edge is below kScreenMax, and both atoms lie within
// +-kScreenMax (pos32.w = 1).
constexpr float kScreenBand = 0.05f;
struct Screen {
    bool on = false;
    float L[3], Li[3], lo2, hi2;
};

__device__ __forceinline__ Screen make_screen(const double* h, const double* hi, bool diag, double rc2) {
    Screen sc;
    const double rc = sqrt(rc2);
    sc.on = diag && 0.5 * fmin(fabs(h[0]), fmin(fabs(h[4]), fabs(h[8]))) > rc + 1.0 &&
            fmax(fabs(h[0]), fmax(fabs(h[4]), fabs(h[8]))) < kScreenMax;
    for (int a = 0; a < 3; a++) { sc.L[a] = (float)h[4 * a]; sc.Li[a] = (float)hi[4 * a]; }
    sc.lo2 = (float)rc2 - kScreenBand;
    sc.hi2 = (float)rc2 + kScreenBand;
    return sc;
}

// Emits the accepted candidates j = c0 .. c1-1 (ascending) of the row being
// built; `emitted` counts every accepted candidate, entries past `cap` are
// not stored.
__device__ __forceinline__ void emit_range(const double* __restrict__ pos, const float4* __restrict__ pos32, int i,
                                           int c0, int c1, const double* h, const double* hi, bool diag, double rc2,
                                           const Screen& sc, bool intra, int cap, int* __restrict__ row,
                                           int& emitted, int lane) {
    const float4 pi = sc.on ? pos32[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    for (int b = c0; b < c1; b += 32) {
        const int j = b + lane;
        bool ok = j < c1 && (!intra || j != i);
        if (ok) {
            const float4 q = sc.on ? pos32[j] : make_float4(0.f, 0.f, 0.f, 0.f);
            if (sc.on && pi.w != 0.0f && q.w != 0.0f) {
                float dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
                dx = fmaf(-sc.L[0], rintf(dx * sc.Li[0]), dx);
                dy = fmaf(-sc.L[1], rintf(dy * sc.Li[1]), dy);
                dz = fmaf(-sc.L[2], rintf(dz * sc.Li[2]), dz);
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                ok = r2 < sc.lo2 ? true : (r2 > sc.hi2 ? false : pair_in(pos, i, j, h, hi, diag, rc2));
            } else {
                ok = pair_in(pos, i, j, h, hi, diag, rc2);
            }
        }
        const unsigned m = __ballot_sync(kFull, ok);
        const int k = emitted + __popc(m & ((1u << lane) - 1u));
        if (ok && k < cap) row[k] = j;
        emitted += __popc(m);
    }
}

// Rows of the intermolecular half list (MODE 0) or the intramolecular list
// (MODE 1); one warp per atom.
template <int MODE>
__global__ void __launch_bounds__(256)
k_mol_rows(const double* __restrict__ pos, const double* __restrict__ hh, int n, const int* __restrict__ off,
           const int* __restrict__ amol, const int* __restrict__ npart, const int* __restrict__ part, int pmax,
           const float4* __restrict__ pos32, double rc2, int cap, int* __restrict__ cnt, int* __restrict__ list,
           int* __restrict__ dropped, const int* __restrict__ flag) {
    if (MODE == 0 && flag[0] == 0) return;
    __shared__ double s_hh[18];
    if (threadIdx.x < 18) s_hh[threadIdx.x] = hh[threadIdx.x];
    __syncthreads();
    const double* h = s_hh;
    const double* hi = s_hh + 9;
    const bool diag = diag_cell(h, hi);
    // intramolecular rows are short: no screen
    Screen sc = make_screen(h, hi, diag, rc2);
    if (MODE == 1) sc.on = false;
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < n; i += gridDim.x * wpb) {
        const int A = amol[i];
        int* row = list + (size_t)i * cap;
        int emitted = 0;
        if (MODE == 1) {
            emit_range(pos, pos32, i, off[A], off[A + 1], h, hi, diag, rc2, sc, true, cap, row, emitted, lane);
        } else {
            const int np = npart[A];
            for (int p = 0; p < np; p++) {
                const int B = part[(size_t)A * pmax + p];
                if (B < A) continue;
                emit_range(pos, pos32, i, off[B], off[B + 1], h, hi, diag, rc2, sc, false, cap, row, emitted, lane);
            }
        }
        if (lane == 0) {
            cnt[i] = emitted < cap ? emitted : cap;
            if (emitted > cap && dropped) atomicAdd(dropped, emitted - cap);
        }
    }
}

// Half-list rows when every molecule has S atoms: atom i's candidates are the
// atoms of its partner molecules above its own, ascending, i.e. candidate k
// is atom k mod S of the (k div S)-th such partner.  The partners' first atoms
// go to shared memory once per atom, and the warp walks the candidates as one
// sequence, 32 * kFlatU at a time, so each lane has kFlatU candidate loads in
// flight instead of a dependent partner lookup per molecule.  Same test, order
// and truncation as k_mol_rows<0>.  k div S is (k + 0.5) * fl(1/S) truncated:
// the quotient's fractional part stays 0.5/S from an integer, and the FP32
// product's relative error (<= 2^-23) cannot cross that for k < 4e6.
// PAIRED (32 <= S <= 64): the walk goes by partner instead, two 32-lane
// slices per partner (atoms 0-31, 32-63; lanes past S idle), kFlatU / 2
// partners at a time -- no quotient per candidate -- and the ballot of the
// kept entries of slice h of the p-th higher partner is stored as word 2 p + h
// of the atom's candidate bitmap, bm[(A * 2 pmax + 2 p + h) * S + i - off[A]],
// from which k_mol_incoming forms the full rows.
constexpr int kFlatU = 4;
constexpr int kFlatWarps = 8;

template <bool PAIRED>
__device__ __forceinline__ void mol_half_flat_body(const double* __restrict__ pos, const double* __restrict__ hh,
                                                   int n, const int* __restrict__ off, const int* __restrict__ amol,
                                                   const int* __restrict__ npart, const int* __restrict__ part,
                                                   int pmax, int S, const float4* __restrict__ pos32, double rc2,
                                                   int cap, int* __restrict__ cnt, int* __restrict__ list,
                                                   int* __restrict__ dropped, const int* __restrict__ flag,
                                                   unsigned* __restrict__ bm, int blk, int nblk) {
    if (flag[0] == 0) return;
    __shared__ double s_hh[18];
    __shared__ int s_start[kFlatWarps][kMolPartners];
    if (threadIdx.x < 18) s_hh[threadIdx.x] = hh[threadIdx.x];
    __syncthreads();
    const double* h = s_hh;
    const double* hi = s_hh + 9;
    const bool diag = diag_cell(h, hi);
    const Screen sc = make_screen(h, hi, diag, rc2);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    int* st = s_start[w];
    const float invS = 1.0f / (float)S;
    for (int i = blk * kFlatWarps + w; i < n; i += nblk * kFlatWarps) {
        const int A = amol[i];
        const int np = npart[A];
        const int* pa = part + (size_t)A * pmax;
        int nup = 0;
        for (int q0 = 0; q0 < np; q0 += 32) {
            const int q = q0 + lane;
            const int B = q < np ? pa[q] : -1;
            const bool up = B > A;
            const unsigned m = __ballot_sync(kFull, up);
            if (up) st[nup + __popc(m & below)] = off[B];
            nup += __popc(m);
        }
        __syncwarp();
        const int ncand = nup * S;
        const float4 pi = pos32[i];
        const bool screen = sc.on && pi.w != 0.0f;
        int* row = list + (size_t)i * cap;
        int emitted = 0;
        unsigned* bmA = PAIRED ? bm + (size_t)A * 2 * pmax * S + (i - off[A]) : nullptr;
        const int nit = PAIRED ? nup : ncand;
        for (int k0 = 0; k0 < nit; k0 += PAIRED ? kFlatU / 2 : 32 * kFlatU) {
            int jj[kFlatU];
            float4 q[kFlatU];
#pragma unroll
            for (int u = 0; u < kFlatU; u++) {
                jj[u] = -1;
                if (PAIRED) {
                    const int p = k0 + (u >> 1), a = ((u & 1) << 5) + lane;
                    if (p < nup && a < S) jj[u] = st[p] + a;
                } else {
                    const int k = k0 + 32 * u + lane;
                    if (k < ncand) {
                        const int pk = (int)(((float)k + 0.5f) * invS);
                        jj[u] = st[pk] + (k - pk * S);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kFlatU; u++) q[u] = jj[u] >= 0 ? pos32[jj[u]] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int u = 0; u < kFlatU; u++) {
                // FP32 screen on every lane (no divergence); the exact FP64
                // test runs, warp-uniformly, only in slices where some lane
                // is in the band, off the screen or without an FP32 copy
                const bool valid = jj[u] >= 0;
                float dx = q[u].x - pi.x, dy = q[u].y - pi.y, dz = q[u].z - pi.z;
                dx = fmaf(-sc.L[0], rintf(dx * sc.Li[0]), dx);
                dy = fmaf(-sc.L[1], rintf(dy * sc.Li[1]), dy);
                dz = fmaf(-sc.L[2], rintf(dz * sc.Li[2]), dz);
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                const bool fast = screen && q[u].w != 0.0f;
                bool ok = valid && fast && r2 < sc.lo2;
                const bool exact = valid && !(fast && (r2 < sc.lo2 || r2 > sc.hi2));
                if (__any_sync(kFull, exact)) {
                    const bool in = pair_in(pos, i, exact ? jj[u] : i, h, hi, diag, rc2);
                    ok = ok || (exact && in);
                }
                const unsigned m = __ballot_sync(kFull, ok);
                const int kk = emitted + __popc(m & below);
                if (ok && kk < cap) row[kk] = jj[u];
                if (PAIRED) {
                    // the slice's entries that fit in the row (row position < cap)
                    const unsigned kept = __ballot_sync(kFull, ok && kk < cap);
                    const int p = k0 + (u >> 1);
                    if (lane == 0 && p < nup) bmA[(size_t)(2 * p + (u & 1)) * S] = kept;
                }
                emitted += __popc(m);
            }
        }
        __syncwarp();                              // st is refilled for the next atom
        if (lane == 0) {
            cnt[i] = emitted < cap ? emitted : cap;
            if (emitted > cap && dropped) atomicAdd(dropped, emitted - cap);
        }
    }
}

template <bool PAIRED>
__global__ void __launch_bounds__(32 * kFlatWarps, 3)
k_mol_half_flat(const double* __restrict__ pos, const double* __restrict__ hh, int n, const int* __restrict__ off,
                const int* __restrict__ amol, const int* __restrict__ npart, const int* __restrict__ part, int pmax,
                int S, const float4* __restrict__ pos32, double rc2, int cap, int* __restrict__ cnt,
                int* __restrict__ list, int* __restrict__ dropped, const int* __restrict__ flag,
                unsigned* __restrict__ bm) {
    mol_half_flat_body<PAIRED>(pos, hh, n, off, amol, npart, part, pmax, S, pos32, rc2, cap, cnt, list, dropped, flag,
                               bm, blockIdx.x, gridDim.x);
}

// First index of a partner >= key in an ascending partner list.
__device__ __forceinline__ int lower_bound_part(const int* pa, int n, int key) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (pa[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// For each lower partner A = part[B][q] (A < B): rev[B][q] = the position p
// of B among the higher partners of A, whose kept-entry ballots are words
// 2 p and 2 p + 1 of each A atom's candidate bitmap.  One warp per
// molecule, binary searches per lane.  The lists are ascending, and symmetric
// (the pair test is odd in the centre difference and symmetric in the radii);
// should B be missing all the same, the molecule builder is switched off for
// this build (flag[0] = 0) and the cell-list path builds.
__device__ __forceinline__ void mol_rev_body(int M, const int* __restrict__ npart, const int* __restrict__ part,
                                             int pmax, int* __restrict__ rev, int* __restrict__ flag, int blk) {
    if (flag[0] == 0) return;
    const int lane = threadIdx.x & 31;
    const int B = (blk * blockDim.x + threadIdx.x) >> 5;
    if (B >= M) return;
    const int nb = npart[B];
    for (int q = lane; q < nb; q += 32) {
        const int A = part[(size_t)B * pmax + q];
        if (A > B) break;                              // ascending: the rest are higher
        const int* pa = part + (size_t)A * pmax;
        const int na = npart[A];
        const int at = lower_bound_part(pa, na, B);
        rev[(size_t)B * pmax + q] = at - lower_bound_part(pa, na, A);
        if (at >= na || pa[at] != B) atomicExch(&flag[0], 0);
    }
}

__global__ void k_mol_rev(int M, const int* __restrict__ npart, const int* __restrict__ part, int pmax,
                          int* __restrict__ rev, int* __restrict__ flag) {
    mol_rev_body(M, npart, part, pmax, rev, flag, blockIdx.x);
}

// Full LJ rows from the candidate bitmaps of the partner-aligned walk
// (k_mol_half_flat<true>), for equal molecules of S atoms (32 <= S <= 64,
// off[A] = A S): atom j = B S + jb is in the kept row of i = A S + ia (A < B)
// iff bit jb mod 32 of word 2 rev[B][q] + jb div 32 of i's bitmap is set.
// Two blocks per molecule B, one per half of its atoms (jb < 32, jb >= 32):
// the half's word of every atom of A is staged in shared memory for up to
// kInChunk lower partners at a time, then warp w emits the rows of atoms
// jb = 32 h + w + 8 t: for each lower partner A (ascending) a ballot over A's
// atoms gives the entries in ascending order.  Row j thus holds the atoms
// i < j whose kept row lists j, ascending, then j's own row -- the rows the
// transpose (nlist_transpose) builds, without atomics or a sort.  The own rows
// are copied with 8 loads in flight per lane.
constexpr int kInChunk = 32;
constexpr int kInWarps = 8;
constexpr int kInAtoms = 32 / kInWarps;               // atoms per warp

__device__ __forceinline__ void mol_incoming_body(int M, int S, const int* __restrict__ npart,
                                                  const int* __restrict__ part, int pmax, const int* __restrict__ rev,
                                                  int W, const unsigned* __restrict__ bm, int cap,
                                                  const int* __restrict__ cnt, const int* __restrict__ list,
                                                  int* __restrict__ in_cnt, int* __restrict__ in_list, int in_cap,
                                                  DevErr* err, const int* __restrict__ flag, int blk, int nblk) {
    if (flag[0] == 0) return;
    __shared__ int s_a[kMolPartners];                 // lower partners, ascending
    __shared__ int s_b[kMolPartners];                 // bitmap word of the half's atoms
    __shared__ unsigned s_bits[kInChunk][64];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    const int lim = in_cap - cap;
    for (int g = blk; g < 2 * M; g += nblk) {
        const int B = g >> 1, h0 = (g & 1) * 32;
        const int nh = S - h0 < 32 ? S - h0 : 32;    // atoms in this half (0 when S = 32, h0 = 32)
        if (nh <= 0) continue;
        int mo[kInAtoms];
#pragma unroll
        for (int t = 0; t < kInAtoms; t++) {
            const int jb = w + kInWarps * t;
            mo[t] = jb < nh ? cnt[B * S + h0 + jb] : 0;
        }
        const int np = npart[B];
        bool low = false;
        for (int q = threadIdx.x; q < np; q += blockDim.x) {     // np <= kMolPartners
            const int A = part[(size_t)B * pmax + q];
            if (A < B) {
                low = true;
                s_a[q] = A;
                s_b[q] = 2 * rev[(size_t)B * pmax + q] + (h0 >> 5);
            }
        }
        const int nlow = __syncthreads_count(low);    // ascending: the lower partners come first
        int em[kInAtoms];
#pragma unroll
        for (int t = 0; t < kInAtoms; t++) em[t] = 0;
        for (int c0 = 0; c0 < nlow; c0 += kInChunk) {
            const int nc = nlow - c0 < kInChunk ? nlow - c0 : kInChunk;
            for (int x = threadIdx.x; x < nc * S; x += blockDim.x) {
                const int c = x / S, ia = x - c * S;
                s_bits[c][ia] = bm[((size_t)s_a[c0 + c] * W + s_b[c0 + c]) * S + ia];
            }
            __syncthreads();
            for (int c = 0; c < nc; c++) {
                const int a0 = s_a[c0 + c] * S;
                const unsigned w0 = s_bits[c][lane], w1 = lane + 32 < S ? s_bits[c][lane + 32] : 0u;
#pragma unroll
                for (int t = 0; t < kInAtoms; t++) {
                    const int jb = w + kInWarps * t;
                    if (jb < nh) {
                        const bool ok0 = (w0 >> jb) & 1u;
                        const bool ok1 = (w1 >> jb) & 1u;
                        const unsigned m0 = __ballot_sync(kFull, ok0), m1 = __ballot_sync(kFull, ok1);
                        int* row = in_list + (size_t)(B * S + h0 + jb) * in_cap;
                        const int p0 = em[t] + __popc(m0 & below);
                        const int p1 = em[t] + __popc(m0) + __popc(m1 & below);
                        if (ok0 && p0 < lim) row[p0] = a0 + lane;
                        if (ok1 && p1 < lim) row[p1] = a0 + lane + 32;
                        em[t] += __popc(m0) + __popc(m1);
                    }
                }
            }
            __syncthreads();                          // s_bits is restaged
        }
        // own rows after the incoming entries
        int mmax = 0;
#pragma unroll
        for (int t = 0; t < kInAtoms; t++) mmax = mo[t] > mmax ? mo[t] : mmax;
        for (int k0 = lane; k0 < mmax; k0 += 64) {
            int v[kInAtoms][2];
#pragma unroll
            for (int t = 0; t < kInAtoms; t++)
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const int k = k0 + 32 * u;
                    v[t][u] = k < mo[t] ? list[(size_t)(B * S + h0 + w + kInWarps * t) * cap + k] : 0;
                }
#pragma unroll
            for (int t = 0; t < kInAtoms; t++) {
                const int kept = em[t] < lim ? em[t] : lim;
                int* row = in_list + (size_t)(B * S + h0 + w + kInWarps * t) * in_cap + kept;
#pragma unroll
                for (int u = 0; u < 2; u++)
                    if (k0 + 32 * u < mo[t]) row[k0 + 32 * u] = v[t][u];
            }
        }
#pragma unroll
        for (int t = 0; t < kInAtoms; t++) {
            const int jb = w + kInWarps * t;
            if (lane == 0 && jb < nh) {
                const int j = B * S + h0 + jb;
                in_cnt[j] = (em[t] < lim ? em[t] : lim) + mo[t];
                if (em[t] > lim && atomicCAS(&err->code, FMD_OK, FMD_ERR_CAPACITY) == FMD_OK) {
                    err->where = K_TRANSPOSE; err->index = j; err->value = em[t];
                }
            }
        }
        __syncthreads();                              // s_a, s_b are refilled
    }
}

__global__ void __launch_bounds__(32 * kInWarps)
k_mol_incoming(int M, int S, const int* __restrict__ npart, const int* __restrict__ part, int pmax,
               const int* __restrict__ rev, int W, const unsigned* __restrict__ bm, int cap,
               const int* __restrict__ cnt, const int* __restrict__ list, int* __restrict__ in_cnt,
               int* __restrict__ in_list, int in_cap, DevErr* err, const int* __restrict__ flag) {
    mol_incoming_body(M, S, npart, part, pmax, rev, W, bm, cap, cnt, list, in_cnt, in_list, in_cap, err, flag,
                      blockIdx.x, gridDim.x);
}

constexpr int kRowBlocksMol = kSMs * 8;

// ------------------------------------------------------- replica batches --
// Block b of a batched launch serves replica r (off[r] <= b < off[r + 1]) as
// its local block b - off[r] of off[r + 1] - off[r].
__device__ __forceinline__ int rep_of(const int* __restrict__ off, int R, int b) {
    int lo = 0, hi = R - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Per replica: h^-1 (as inv9_launch) and the pruned rows marked stale (as
// lj_prune_mark after a build).
__global__ void k_b_inv9(const MolRep* __restrict__ reps, int R) {
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        inv9(reps[r].hh, reps[r].hh + 9);
        if (reps[r].prune_words) *reps[r].prune_words = kPruneMark;
    }
}

__global__ void k_b_mol_centre(const MolRep* __restrict__ reps, const int* __restrict__ off, int R) {
    const int r = rep_of(off, R, blockIdx.x);
    const MolRep& q = reps[r];
    mol_centre_body(q.pos, q.hh, q.m.off, q.m.M, q.m.cen, q.m.rad, q.m.pos32, q.m.flag, blockIdx.x - off[r]);
}

__global__ void k_b_mol_pairs(const MolRep* __restrict__ reps, const int* __restrict__ off, int R) {
    const int r = rep_of(off, R, blockIdx.x);
    const MolRep& q = reps[r];
    mol_pairs_body(q.hh, q.m.M, q.m.cen, q.m.rad, q.rc, q.m.pmax, q.m.npart, q.m.part, q.m.flag, blockIdx.x - off[r]);
}

__global__ void k_b_mol_decide(const MolRep* __restrict__ reps, int R) {
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        const double* hh = reps[r].hh;
        int* flag = reps[r].m.flag;
        flag[0] = (diag_cell(hh, hh + 9) && flag[1] == 0) ? 1 : 0;
    }
}

__global__ void k_b_mol_rev(const MolRep* __restrict__ reps, const int* __restrict__ off, int R) {
    const int r = rep_of(off, R, blockIdx.x);
    const MolRep& q = reps[r];
    mol_rev_body(q.m.M, q.m.npart, q.m.part, q.m.pmax, q.m.rev, q.m.flag, blockIdx.x - off[r]);
}

// Sets the fallback's conditional when some replica's molecule path was
// rejected (by the decision or the partner-symmetry check).
__global__ void k_b_mol_cond(const MolRep* __restrict__ reps, int R, cudaGraphConditionalHandle cond) {
    int need = 0;
    for (int r = threadIdx.x; r < R; r += blockDim.x) need |= reps[r].m.flag[0] == 0;
    if (__syncthreads_or(need) && threadIdx.x == 0) cudaGraphSetConditional(cond, 1u);
}

__global__ void __launch_bounds__(32 * kFlatWarps, 3)
k_b_mol_half_flat(const MolRep* __restrict__ reps, const int* __restrict__ off, int R) {
    const int r = rep_of(off, R, blockIdx.x);
    const MolRep& q = reps[r];
    mol_half_flat_body<true>(q.pos, q.hh, q.m.n, q.m.off, q.m.amol, q.m.npart, q.m.part, q.m.pmax, q.m.usize,
                             q.m.pos32, q.rc2, q.cap, q.cnt, q.list, q.dropped, q.m.flag, q.m.bm,
                             blockIdx.x - off[r], off[r + 1] - off[r]);
}

__global__ void __launch_bounds__(32 * kInWarps)
k_b_mol_incoming(const MolRep* __restrict__ reps, const int* __restrict__ off, int R) {
    const int r = rep_of(off, R, blockIdx.x);
    const MolRep& q = reps[r];
    mol_incoming_body(q.m.M, q.m.usize, q.m.npart, q.m.part, q.m.pmax, q.m.rev, q.m.words, q.m.bm, q.cap, q.cnt,
                      q.list, q.in_cnt, q.in_list, q.in_cap, q.err, q.m.flag, blockIdx.x - off[r],
                      off[r + 1] - off[r]);
}

}  // namespace

cudaError_t mol_rebuild_batch_pre(const MolBatch& b, cudaGraphConditionalHandle cond, cudaStream_t st,
                                  const char** stage) {
    if (b.R < 1) return cudaSuccess;
    cudaError_t e;
#define FMD_MB_STEP(NAME, LAUNCH)                              \
    do {                                                       \
        if (stage) *stage = NAME;                              \
        LAUNCH;                                                \
        if ((e = cudaGetLastError()) != cudaSuccess) return e; \
    } while (0)
    FMD_MB_STEP("k_b_inv9", (k_b_inv9<<<1, 256, 0, st>>>(b.reps, b.R)));
    FMD_MB_STEP("k_b_mol_centre", (k_b_mol_centre<<<b.nblk_w, 256, 0, st>>>(b.reps, b.off_w, b.R)));
    FMD_MB_STEP("k_b_mol_pairs", (k_b_mol_pairs<<<b.nblk_w, 256, 0, st>>>(b.reps, b.off_w, b.R)));
    FMD_MB_STEP("k_b_mol_decide", (k_b_mol_decide<<<1, 256, 0, st>>>(b.reps, b.R)));
    FMD_MB_STEP("k_b_mol_rev", (k_b_mol_rev<<<b.nblk_w, 256, 0, st>>>(b.reps, b.off_w, b.R)));
    FMD_MB_STEP("k_b_mol_cond", (k_b_mol_cond<<<1, 256, 0, st>>>(b.reps, b.R, cond)));
#undef FMD_MB_STEP
    return cudaSuccess;
}

cudaError_t mol_rebuild_batch_rows(const MolBatch& b, cudaStream_t st) {
    if (b.R < 1) return cudaSuccess;
    k_b_mol_half_flat<<<b.nblk_rows, 32 * kFlatWarps, 0, st>>>(b.reps, b.off_rows, b.R);
    k_b_mol_incoming<<<b.nblk_in, 32 * kInWarps, 0, st>>>(b.reps, b.off_in, b.R);
    return cudaGetLastError();
}

namespace {
}  // namespace

cudaError_t mol_lists_alloc(MolLists& m, int n, const int* mol_id_host, const DevAlloc& da) {
    m = MolLists();
    if (n <= 0 || !mol_id_host) return cudaSuccess;
    // contiguous molecules: each id forms one run
    std::vector<int> off;
    off.push_back(0);
    for (int k = 1; k < n; k++)
        if (mol_id_host[k] != mol_id_host[k - 1]) off.push_back(k);
    off.push_back(n);
    const int M = (int)off.size() - 1;
    {
        std::vector<int> ids;
        for (int a = 0; a < M; a++) ids.push_back(mol_id_host[off[a]]);
        std::sort(ids.begin(), ids.end());
        for (int a = 1; a < M; a++)
            if (ids[a] == ids[a - 1]) return cudaSuccess;     // an id in two runs: not contiguous
    }
    std::vector<int> amol(n);
    for (int a = 0; a < M; a++)
        for (int k = off[a]; k < off[a + 1]; k++) amol[k] = a;
    m.M = M;
    m.pmax = std::min(M, kMolPartners);
    for (int a = 0; a < M; a++) m.max_atoms = std::max(m.max_atoms, off[a + 1] - off[a]);
    m.usize = m.max_atoms;
    for (int a = 0; a < M; a++)
        if (off[a + 1] - off[a] != m.usize) m.usize = 0;
    m.masks = m.usize >= 32 && m.usize <= 64;
    m.words = 2 * m.pmax;
    cudaError_t e;
    auto A = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = da(p, bytes);
    };
    e = cudaSuccess;
    m.ext = da.fn != nullptr;
    A((void**)&m.off, sizeof(int) * (M + 1));
    A((void**)&m.amol, sizeof(int) * n);
    A((void**)&m.cen, sizeof(double) * 3 * M);
    A((void**)&m.rad, sizeof(double) * M);
    A((void**)&m.pos32, sizeof(float4) * n);
    if (m.masks) {
        A((void**)&m.bm, sizeof(unsigned) * (size_t)M * m.words * m.usize);
        A((void**)&m.rev, sizeof(int) * (size_t)M * m.pmax);
    }
    A((void**)&m.npart, sizeof(int) * M);
    A((void**)&m.part, sizeof(int) * (size_t)M * m.pmax);
    A((void**)&m.flag, sizeof(int) * 2);
    if (e == cudaSuccess) e = cudaMemcpy(m.off, off.data(), sizeof(int) * (M + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m.amol, amol.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m.flag, 0, sizeof(int) * 2);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);     // before any other stream reads them
    if (e != cudaSuccess) {
        mol_lists_free(m);
        return e;
    }
    m.n = n;
    m.ok = true;
    return cudaSuccess;
}

void mol_lists_free(MolLists& m) {
    if (m.ext) {
        m = MolLists();
        return;
    }
    cudaFree(m.off); cudaFree(m.amol); cudaFree(m.cen); cudaFree(m.rad); cudaFree(m.pos32); cudaFree(m.bm);
    cudaFree(m.rev); cudaFree(m.npart); cudaFree(m.part);
    cudaFree(m.flag);
    m = MolLists();
}

cudaError_t mol_partners(MolLists& m, const double* pos, const double* hh, double rc, cudaStream_t st) {
    const int wblocks = (m.M * 32 + 255) / 256;
    k_mol_centre<<<wblocks, 256, 0, st>>>(pos, hh, m.off, m.M, m.cen, m.rad, m.pos32, m.flag);
    k_mol_pairs<<<wblocks, 256, 0, st>>>(hh, m.M, m.cen, m.rad, rc, m.pmax, m.npart, m.part, m.flag);
    k_mol_decide<<<1, 32, 0, st>>>(hh, m.flag);
    if (m.masks) k_mol_rev<<<wblocks, 256, 0, st>>>(m.M, m.npart, m.part, m.pmax, m.rev, m.flag);
    return cudaGetLastError();
}

cudaError_t mol_rows_intra(const MolLists& m, const double* pos, const double* hh, double rc2, int cap, int* cnt,
                           int* list, int* dropped, cudaStream_t st) {
    k_mol_rows<1><<<kRowBlocksMol, 256, 0, st>>>(pos, hh, m.n, m.off, m.amol, m.npart, m.part, m.pmax, m.pos32, rc2,
                                                 cap, cnt, list, dropped, m.flag);
    return cudaGetLastError();
}

cudaError_t mol_rows_half(const MolLists& m, const double* pos, const double* hh, double rc2, int cap, int* cnt,
                          int* list, int* dropped, cudaStream_t st) {
    if (m.masks) {
        k_mol_half_flat<true><<<kRowBlocksMol, 32 * kFlatWarps, 0, st>>>(pos, hh, m.n, m.off, m.amol, m.npart,
                                                                         m.part, m.pmax, m.usize, m.pos32, rc2, cap,
                                                                         cnt, list, dropped, m.flag, m.bm);
        return cudaGetLastError();
    }
    if (m.usize > 0) {
        k_mol_half_flat<false><<<kRowBlocksMol, 32 * kFlatWarps, 0, st>>>(pos, hh, m.n, m.off, m.amol, m.npart,
                                                                          m.part, m.pmax, m.usize, m.pos32, rc2, cap,
                                                                          cnt, list, dropped, m.flag, nullptr);
        return cudaGetLastError();
    }
    k_mol_rows<0><<<kRowBlocksMol, 256, 0, st>>>(pos, hh, m.n, m.off, m.amol, m.npart, m.part, m.pmax, m.pos32, rc2,
                                                 cap, cnt, list, dropped, m.flag);
    return cudaGetLastError();
}

cudaError_t mol_rows_incoming(const MolLists& m, int cap, const int* cnt, const int* list, int* in_cnt,
                              int* in_list, int in_cap, DevErr* err, cudaStream_t st) {
    if (!m.masks) return cudaErrorInvalidValue;
    const int blocks = 2 * m.M < kRowBlocksMol ? 2 * m.M : kRowBlocksMol;
    k_mol_incoming<<<blocks, 32 * kInWarps, 0, st>>>(m.M, m.usize, m.npart, m.part, m.pmax, m.rev, m.words, m.bm,
                                                     cap, cnt, list, in_cnt, in_list, in_cap, err, m.flag);
    return cudaGetLastError();
}

}  // namespace fmd
