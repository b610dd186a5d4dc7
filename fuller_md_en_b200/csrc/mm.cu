// mm.cu -- molecular-mechanics bonded terms and cut Coulomb (MM:378-709,
// MM:766-786).
//
// Bonded terms: one thread per term over the concatenated index space
// [bonds | angles | dihedrals | impropers]; forces scattered with FP64
// atomics into an accumulator that the LJ gather kernel folds into F and
// clears.  Sign conventions follow the reference exactly, including the bond
// and angle forces that equal +grad E (MM:389-398, MM:468-491), unless the
// topology is marked physical: then those two are negated, and so are the
// torsions' projection terms on their middle atoms (torsion()), and every MM
// force is -grad E (the reference path multiplies by 1.0: its arithmetic is
// unchanged).  Energies and
// the bond diagonal virial go to per-block partials.
//
// Coulomb: all pairs of different molecules within 3 sigma, gathered per atom
// through shared-memory tiles (no atomics); energy counted for j>i only.  The
// reference runs it serially only when some charge is nonzero (MM:1110-1111).
#include <algorithm>
#include <cmath>
#include "kernels.h"
#include "geom.cuh"
#include "step.h"

namespace fmd {
namespace {

__device__ __forceinline__ void load_cell(const double* __restrict__ hh, double* h, double* hi) {
#pragma unroll
    for (int k = 0; k < 9; k++) { h[k] = hh[k]; hi[k] = hh[9 + k]; }
}

__device__ __forceinline__ void vec(const double* __restrict__ pos, int a, int b, const double* h,
                                    const double* hi, double& x, double& y, double& z) {
    x = __dsub_rn(pos[3 * b], pos[3 * a]);
    y = __dsub_rn(pos[3 * b + 1], pos[3 * a + 1]);
    z = __dsub_rn(pos[3 * b + 2], pos[3 * a + 2]);
    mimg(x, y, z, hi, h);
}

__device__ __forceinline__ void add3(double* F, int i, double x, double y, double z) {
    atomicAdd(&F[3 * i], x);
    atomicAdd(&F[3 * i + 1], y);
    atomicAdd(&F[3 * i + 2], z);
}

// Torsion of atoms a1-a2-a3-a4 (MM:503-601); returns the energy.  The forces
// on a1 and a4 are -dE/dphi dphi/dr; on the middle atoms the reference adds
// the projections ci f1 - ck f4 with the opposite sign to the gradient's
// (b1 = r2 - r1 where the gradient formula's vector is r1 - r2), so they are
// not -grad E.  sg = -1 (physical forces) negates ci and ck, giving -grad E;
// sg = 1 is the reference's arithmetic exactly.
__device__ double torsion(double* F, const double* __restrict__ pos, const double* h, const double* hi,
                          int a1, int a2, int a3, int a4, int mult, double vn, double gamma, double sg) {
    double b1x, b1y, b1z, b2x, b2y, b2z, b3x, b3y, b3z;
    vec(pos, a1, a2, h, hi, b1x, b1y, b1z);
    vec(pos, a2, a3, h, hi, b2x, b2y, b2z);
    vec(pos, a3, a4, h, hi, b3x, b3y, b3z);
    const double mx = b1y * b2z - b1z * b2y, my = b1z * b2x - b1x * b2z, mz = b1x * b2y - b1y * b2x;
    const double nx = b2y * b3z - b2z * b3y, ny = b2z * b3x - b2x * b3z, nz = b2x * b3y - b2y * b3x;
    const double mm = mx * mx + my * my + mz * mz, nn = nx * nx + ny * ny + nz * nz;
    if (mm < 1e-20 || nn < 1e-20) return 0.0;
    const double imm = 1.0 / mm, inn = 1.0 / nn;
    const double b2len = sqrt(b2x * b2x + b2y * b2y + b2z * b2z);
    const double rmn = sqrt(mm * nn);
    double cosphi = (mx * nx + my * ny + mz * nz) / rmn;
    cosphi = cosphi > 1.0 ? 1.0 : (cosphi < -1.0 ? -1.0 : cosphi);
    const double b1b2 = b1x * b2x + b1y * b2y + b1z * b2z;
    const double b2b3 = b2x * b3x + b2y * b3y + b2z * b3z;
    const double sinphi = (mx * b3x + my * b3y + mz * b3z) * b2len / rmn;
    const double phi = atan2(sinphi, cosphi);
    const double e = 0.5 * vn * (1.0 + cos(mult * phi - gamma));
    const double dphi = -0.5 * vn * mult * sin(mult * phi - gamma);
    const double g1 = dphi * b2len * imm, g4 = -dphi * b2len * inn;
    const double f1x = g1 * mx, f1y = g1 * my, f1z = g1 * mz;
    const double f4x = g4 * nx, f4y = g4 * ny, f4z = g4 * nz;
    const double ci = sg * (b1b2 / (b2len * b2len)), ck = sg * (b2b3 / (b2len * b2len));
    add3(F, a1, f1x, f1y, f1z);
    add3(F, a2, -f1x + ci * f1x - ck * f4x, -f1y + ci * f1y - ck * f4y, -f1z + ci * f1z - ck * f4z);
    add3(F, a3, -f4x - ci * f1x + ck * f4x, -f4y - ci * f1y + ck * f4y, -f4z - ci * f1z + ck * f4z);
    add3(F, a4, f4x, f4y, f4z);
    return e;
}

// Terms blk*blockDim + tid, strided by nblk*blockDim; partials into part[blk].
__device__ __forceinline__ void mm_bonded_body(const MMTopoDev& t, const double* __restrict__ pos,
                                               const double* __restrict__ hh, double* __restrict__ F,
                                               double* __restrict__ part, int blk, int nblk, double* sm) {
    double h[9], hi[9];
    load_cell(hh, h, hi);
    double acc[kMMNV];   // Eb Ea Ed Ei W00 W11 W22
#pragma unroll
    for (int k = 0; k < kMMNV; k++) acc[k] = 0.0;
    const double sg = t.physical ? -1.0 : 1.0;
    const int total = t.nb + t.nang + t.ndih + t.nimp;
    for (int q = blk * blockDim.x + threadIdx.x; q < total; q += nblk * blockDim.x) {
        if (q < t.nb) {                                           // MM:384-447
            const int b = q, i = t.b_i0[b], j = t.b_i1[b];
            double dx, dy, dz;
            vec(pos, i, j, h, hi, dx, dy, dz);
            const double r = sqrt(norm2_rn(dx, dy, dz));
            if (r < 1e-10) continue;
            const double dr = r - t.b_r0[b];
            acc[0] += 0.5 * t.b_kb[b] * dr * dr;
            const double fm = sg * (-t.b_kb[b] * dr / r);
            const double fx = fm * dx, fy = fm * dy, fz = fm * dz;
            add3(F, i, fx, fy, fz);
            add3(F, j, -fx, -fy, -fz);
            acc[4] += dx * fx; acc[5] += dy * fy; acc[6] += dz * fz;
        } else if (q < t.nb + t.nang) {                           // MM:455-492
            const int a = q - t.nb, i = t.a_i0[a], j = t.a_i1[a], k = t.a_i2[a];
            double u0, u1, u2, v0, v1, v2;
            vec(pos, j, i, h, hi, u0, u1, u2);
            vec(pos, j, k, h, hi, v0, v1, v2);
            const double du = sqrt(u0 * u0 + u1 * u1 + u2 * u2), dv = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
            if (du < 1e-10 || dv < 1e-10) continue;
            double c = (u0 * v0 + u1 * v1 + u2 * v2) / (du * dv);
            c = c > 0.999999 ? 0.999999 : (c < -0.999999 ? -0.999999 : c);
            const double th = acos(c), dth = th - t.a_th0[a];
            acc[1] += 0.5 * t.a_kth[a] * dth * dth;
            const double s = sqrt(1.0 - c * c + 1e-30);
            const double dV = sg * (-t.a_kth[a] * dth / s);
            const double uv = du * dv, uu = du * du, vv = dv * dv;
            const double fi0 = dV * (v0 / uv - c * u0 / uu), fi1 = dV * (v1 / uv - c * u1 / uu),
                         fi2 = dV * (v2 / uv - c * u2 / uu);
            const double fk0 = dV * (u0 / uv - c * v0 / vv), fk1 = dV * (u1 / uv - c * v1 / vv),
                         fk2 = dV * (u2 / uv - c * v2 / vv);
            add3(F, i, fi0, fi1, fi2);
            add3(F, k, fk0, fk1, fk2);
            add3(F, j, -(fi0 + fk0), -(fi1 + fk1), -(fi2 + fk2));
        } else if (q < t.nb + t.nang + t.ndih) {                  // MM:500-602
            const int d = q - t.nb - t.nang;
            acc[2] += torsion(F, pos, h, hi, t.d_i0[d], t.d_i1[d], t.d_i2[d], t.d_i3[d], t.d_mult[d],
                              t.d_vn[d], t.d_gamma[d], sg);
        } else {                                                  // MM:610-709, order c1,c0,c2,c3
            const int p = q - t.nb - t.nang - t.ndih;
            acc[3] += torsion(F, pos, h, hi, t.m_i1[p], t.m_i0[p], t.m_i2[p], t.m_i3[p], 2, t.m_ki[p],
                              t.m_gamma[p], sg);
        }
    }
    block_sum_store<kMMNV>(acc, sm, part + (size_t)blk * kMMNV);
}

__global__ void __launch_bounds__(128)
k_mm_bonded(MMTopoDev t, const double* __restrict__ pos, const double* __restrict__ hh,
            double* __restrict__ F, double* __restrict__ part) {
    __shared__ double sm[32 * kMMNV];
    mm_bonded_body(t, pos, hh, F, part, blockIdx.x, gridDim.x, sm);
}

template <int NT>
__global__ void __launch_bounds__(NT) k_b_mm_bonded(const StepArrays* __restrict__ As, const int* __restrict__ off,
                                                    int R) {
    __shared__ double sm[32 * kMMNV];
    const int r = batch_rep(off, R, blockIdx.x);
    const StepArrays& a = As[r];
    mm_bonded_body(a.topo, a.pos, a.S->h, a.Facc, a.part_f1, blockIdx.x - off[r], off[r + 1] - off[r], sm);
}

constexpr int kTile = 128;

__global__ void __launch_bounds__(kTile)
k_coulomb(const double* __restrict__ pos, const double* __restrict__ hh, const double* __restrict__ charge,
          const int* __restrict__ mol_id, int na, double* __restrict__ F, double* __restrict__ part) {
    __shared__ double sx[kTile], sy[kTile], sz[kTile], sq[kTile];
    __shared__ int smol[kTile];
    __shared__ double sm[32];
    double h[9], hi[9];
    load_cell(hh, h, hi);
    const double kc = 14.3996, rcut = 3.0 * 3.431, rc2 = rcut * rcut;   // MM:117-118
    double eacc[1] = {0.0};
    for (int base = blockIdx.x * kTile; base < na; base += gridDim.x * kTile) {
        const int i = base + threadIdx.x;
        const bool act = i < na;
        const double px = act ? pos[3 * i] : 0, py = act ? pos[3 * i + 1] : 0, pz = act ? pos[3 * i + 2] : 0;
        const double qi = act ? charge[i] : 0;
        const int mi = act ? mol_id[i] : -1;
        double fx = 0, fy = 0, fz = 0;
        for (int t0 = 0; t0 < na; t0 += kTile) {
            const int jj = t0 + threadIdx.x;
            if (jj < na) {
                sx[threadIdx.x] = pos[3 * jj]; sy[threadIdx.x] = pos[3 * jj + 1]; sz[threadIdx.x] = pos[3 * jj + 2];
                sq[threadIdx.x] = charge[jj]; smol[threadIdx.x] = mol_id[jj];
            }
            __syncthreads();
            const int lim = na - t0 < kTile ? na - t0 : kTile;
            if (act) {
                for (int k = 0; k < lim; k++) {
                    const int j = t0 + k;
                    if (j == i || smol[k] == mi) continue;
                    double dx = __dsub_rn(sx[k], px), dy = __dsub_rn(sy[k], py), dz = __dsub_rn(sz[k], pz);
                    mimg(dx, dy, dz, hi, h);
                    const double r2 = norm2_rn(dx, dy, dz);
                    if (r2 > rc2) continue;
                    const double r = sqrt(r2), qq = kc * qi * sq[k];
                    if (j > i) eacc[0] += qq / r - qq / rcut;
                    const double fm = qq / (r2 * r);
                    fx -= fm * dx; fy -= fm * dy; fz -= fm * dz;
                }
            }
            __syncthreads();
        }
        if (act) { F[3 * i] += fx; F[3 * i + 1] += fy; F[3 * i + 2] += fz; }
    }
    double tot[1];
    block_sum_store<1>(eacc, sm, tot);
    if (threadIdx.x == 0) part[blockIdx.x] = tot[0];
}

// One thread per output term, over [bonds | angles | dihedrals | impropers]
// of all copies.
__global__ void k_mm_replicate(MMTopoDev t, int nmol, int natom, MMTopoOut o) {
    const long long nb = (long long)nmol * t.nb, na = (long long)nmol * t.nang, nd = (long long)nmol * t.ndih,
                    ni = (long long)nmol * t.nimp;
    const long long tot = nb + na + nd + ni;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < tot;
         x += (long long)gridDim.x * blockDim.x) {
        long long y = x;
        if (y < nb) {
            const int m = (int)(y / t.nb), k = (int)(y - (long long)m * t.nb), off = m * natom;
            o.b_i0[y] = t.b_i0[k] + off; o.b_i1[y] = t.b_i1[k] + off;
            o.b_kb[y] = t.b_kb[k]; o.b_r0[y] = t.b_r0[k];
            continue;
        }
        y -= nb;
        if (y < na) {
            const int m = (int)(y / t.nang), k = (int)(y - (long long)m * t.nang), off = m * natom;
            o.a_i0[y] = t.a_i0[k] + off; o.a_i1[y] = t.a_i1[k] + off; o.a_i2[y] = t.a_i2[k] + off;
            o.a_kth[y] = t.a_kth[k]; o.a_th0[y] = t.a_th0[k];
            continue;
        }
        y -= na;
        if (y < nd) {
            const int m = (int)(y / t.ndih), k = (int)(y - (long long)m * t.ndih), off = m * natom;
            o.d_i0[y] = t.d_i0[k] + off; o.d_i1[y] = t.d_i1[k] + off;
            o.d_i2[y] = t.d_i2[k] + off; o.d_i3[y] = t.d_i3[k] + off;
            o.d_vn[y] = t.d_vn[k]; o.d_mult[y] = t.d_mult[k]; o.d_gamma[y] = t.d_gamma[k];
            continue;
        }
        y -= nd;
        const int m = (int)(y / t.nimp), k = (int)(y - (long long)m * t.nimp), off = m * natom;
        o.m_i0[y] = t.m_i0[k] + off; o.m_i1[y] = t.m_i1[k] + off;
        o.m_i2[y] = t.m_i2[k] + off; o.m_i3[y] = t.m_i3[k] + off;
        o.m_ki[y] = t.m_ki[k]; o.m_gamma[y] = t.m_gamma[k];
    }
}

}  // namespace

cudaError_t mm_replicate_launch(const MMTopoDev& mol, int nmol, int natom, const MMTopoOut& out, cudaStream_t st) {
    const long long tot = (long long)nmol * ((long long)mol.nb + mol.nang + mol.ndih + mol.nimp);
    if (tot <= 0) return cudaSuccess;
    const int blocks = (int)std::min<long long>((tot + 255) / 256, kSMs * 16);
    k_mm_replicate<<<blocks, 256, 0, st>>>(mol, nmol, natom, out);
    return cudaGetLastError();
}

cudaError_t mm_bonded_launch(const MMTopoDev& t, const double* pos, const double* hh, double* Facc,
                             double* part, cudaStream_t st) {
    k_mm_bonded<<<kForceBlocks, 128, 0, st>>>(t, pos, hh, Facc, part);
    return cudaGetLastError();
}

cudaError_t batch_mm_bonded_launch(const StepArrays* As, const int* off, int R, int nblocks, int threads,
                                   cudaStream_t st) {
    if (threads == 256) k_b_mm_bonded<256><<<nblocks, 256, 0, st>>>(As, off, R);
    else k_b_mm_bonded<128><<<nblocks, 128, 0, st>>>(As, off, R);
    return cudaGetLastError();
}

cudaError_t mm_coulomb_launch(const double* pos, const double* hh, const double* charge, const int* mol_id,
                              int na, double* Facc, double* part, cudaStream_t st) {
    k_coulomb<<<kForceBlocks, kTile, 0, st>>>(pos, hh, charge, mol_id, na, Facc, part);
    return cudaGetLastError();
}

}  // namespace fmd
