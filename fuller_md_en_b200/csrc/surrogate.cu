// surrogate.cu -- inference path of the learned bond-order potential.
//
//   k_sg_count / k_sg_scan / k_sg_rows   directed bonds (rows), compacted
//   k_sg_desc    32-wide descriptor per row -> BF16 tiles of 128 rows
//   k_sg_mlp     fused 3 x 128 SiLU network on the tensor cores: three
//                forward GEMMs and three gradient-network GEMMs per tile
//                (tcgen05.mma, BF16 operands in shared memory, FP32
//                accumulators in TMEM), giving b and db/dx per row
//   k_sg_force   REBO pair term with b_bar = (b_ij + b_ji)/2 and the
//                reference's three-body construction with db/dr_k
//
// The network and its gradient network never leave the SM: the pre-
// activations z1, z2, z3 stay in TMEM columns [0,384) and the gradient GEMMs
// accumulate in [384,512); each epilogue reads TMEM, applies SiLU or its
// derivative in FP32, and writes the next BF16 operand tile to shared
// memory.  W_l^T is the MN-major view of the same shared-memory image as
// W_l (umma.cuh), so each weight matrix is held once.
#include <cuda_bf16.h>

#include "kernels.h"
#include "rebo_fn.cuh"
#include "sg_dev.cuh"
#include "surrogate.cuh"
#include "umma.cuh"

namespace fmd {
namespace sg {
namespace {

using namespace rebo;
using namespace dev;

// Rows of each atom (bonds kept by the row rule), and their exclusive scan
// within each block of 256 atoms (block totals in bsum); one atom per thread.
constexpr int kScanBlock = 256;

__global__ void __launch_bounds__(kScanBlock)
k_sg_count(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ cnt,
           const int* __restrict__ list, int cap, int na, int* __restrict__ acnt, const int* __restrict__ gate,
           int* __restrict__ aoff, int* __restrict__ bsum) {
    __shared__ int wsum[kScanBlock / 32];
    double h[9], hi[9];
    load_cell(hh, h, hi);
    // A set gate (the plain kernel has taken over) leaves every atom without rows.
    const bool off = gate != nullptr && *gate != 0;
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    int c = 0;
    if (i < na && !off) {
        for (int jn = 0; jn < cnt[i]; jn++) {
            double x, y, z;
            bond_vec(pos, i, list[(size_t)i * cap + jn], h, hi, x, y, z);
            c += bond_kept(sqrt(norm2_rn(x, y, z)));
        }
    }
    if (i < na) acnt[i] = c;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    int before = 0, total = 0;
    for (int k = 0; k < kScanBlock / 32; k++) {
        if (k < wid) before += wsum[k];
        total += wsum[k];
    }
    if (i < na) aoff[i] = before + incl - c;          // block-local exclusive offset
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// Exclusive scan of acnt[0..na) into aoff[0..na]; one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_sg_scan(const int* __restrict__ acnt, int na, int* __restrict__ aoff) {
    __shared__ int sm[1024];
    const int per = (na + 1023) / 1024;
    const int b0 = min((int)threadIdx.x * per, na), b1 = min(b0 + per, na);
    int s = 0;
    for (int c = b0; c < b1; c++) s += acnt[c];
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int t = threadIdx.x >= o ? sm[threadIdx.x - o] : 0;
        __syncthreads();
        sm[threadIdx.x] += t;
        __syncthreads();
    }
    int run = sm[threadIdx.x] - s;
    for (int c = b0; c < b1; c++) {
        aoff[c] = run;
        run += acnt[c];
    }
    if (threadIdx.x == 1023) aoff[na] = sm[1023];
}

__global__ void k_sg_rows(const double* __restrict__ pos, const double* __restrict__ hh,
                          const int* __restrict__ cnt, const int* __restrict__ list, int cap, int na,
                          int* __restrict__ aoff, int* __restrict__ row_i, int* __restrict__ row_s,
                          int* __restrict__ rowid, const int* __restrict__ gate, const int* __restrict__ boff) {
    // global offsets: block-local offset + the block's scanned total
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    const int nblk = (na + kScanBlock - 1) / kScanBlock;
    if (i == 0) aoff[na] = boff[nblk];
    if (i >= na) return;
    const int r0 = aoff[i] + boff[blockIdx.x];
    aoff[i] = r0;
    if (gate != nullptr && *gate != 0) return;
    double h[9], hi[9];
    load_cell(hh, h, hi);
    {
        int r = r0;
        for (int jn = 0; jn < cap; jn++) {
            int id = -1;
            if (jn < cnt[i]) {
                double x, y, z;
                bond_vec(pos, i, list[(size_t)i * cap + jn], h, hi, x, y, z);
                if (bond_kept(sqrt(norm2_rn(x, y, z)))) {
                    id = r++;
                    row_i[id] = i;
                    row_s[id] = jn;
                }
            }
            rowid[(size_t)i * cap + jn] = id;
        }
    }
}

// One thread per row: features, normalisation, BF16 tile row, partner row.
__global__ void k_sg_desc(const double* __restrict__ pos, const double* __restrict__ hh,
                          const int* __restrict__ cnt, const int* __restrict__ list, int cap, int na,
                          const int* __restrict__ aoff, const int* __restrict__ row_i,
                          const int* __restrict__ row_s, const int* __restrict__ rowid, const float* __restrict__ vec,
                          int r_cap, uint16_t* __restrict__ X, int* __restrict__ partner, int* __restrict__ err) {
    double h[9], hi[9];
    load_cell(hh, h, hi);
    const int R = aoff[na];
    const int Rpad = (R + TILE - 1) / TILE * TILE;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < Rpad && r < r_cap; r += gridDim.x * blockDim.x) {
        float x[D];
#pragma unroll
        for (int f = 0; f < D; f++) x[f] = 0.f;
        if (r < R) {
            const int i = row_i[r], j = list[(size_t)i * cap + row_s[r]];
            double dx, dy, dz;
            bond_vec(pos, i, j, h, hi, dx, dy, dz);
            const double rij = sqrt(norm2_rn(dx, dy, dz));
            for (int kn = 0; kn < cnt[i]; kn++) {
                const int k = list[(size_t)i * cap + kn];
                if (k == j) continue;
                double kx, ky, kz;
                bond_vec(pos, i, k, h, hi, kx, ky, kz);
                const double rk = sqrt(norm2_rn(kx, ky, kz));
                if (rk > DMAX_CC) continue;
                const double fk = sw_fc(rk);
                if (fk < 1e-15) continue;
                const float c = (float)clamp1((dx * kx + dy * ky + dz * kz) / (rij * rk));
                float Tr[NR], dTr[NR], Ta[NA], dTa[NA];
                cheb<NR>((float)((rk - RHO_C) / RHO_W), Tr, dTr);
                cheb<NA>(c, Ta, dTa);
#pragma unroll
                for (int a = 0; a < NR; a++)
#pragma unroll
                    for (int b = 0; b < NA; b++) x[a * NA + b] += (float)fk * Tr[a] * Ta[b];
            }
            // partner row (j -> i)
            int p = -1;
            for (int ln = 0; ln < cnt[j]; ln++)
                if (list[(size_t)j * cap + ln] == i) { p = rowid[(size_t)j * cap + ln]; break; }
            if (p < 0) {
                atomicCAS(err, 0, r + 1);
                p = r;
            }
            partner[r] = p;
#pragma unroll
            for (int f = 0; f < D - 1; f++) x[f] = (x[f] - vec[V_M + f]) * vec[V_SINV + f];
            x[D - 1] = 1.f;
        }
        unsigned char* tile = reinterpret_cast<unsigned char*>(X) + (size_t)(r / TILE) * TILE * D * 2;
        const int q = r % TILE;
#pragma unroll
        for (int c8 = 0; c8 < D / 8; c8++) {
            uint4 v;
            v.x = umma::pack_bf16(x[8 * c8 + 0], x[8 * c8 + 1]);
            v.y = umma::pack_bf16(x[8 * c8 + 2], x[8 * c8 + 3]);
            v.z = umma::pack_bf16(x[8 * c8 + 4], x[8 * c8 + 5]);
            v.w = umma::pack_bf16(x[8 * c8 + 6], x[8 * c8 + 7]);
            *reinterpret_cast<uint4*>(tile + umma::il_off(q, 8 * c8, D)) = v;
        }
    }
}

// ------------------------------------------------------------------ network
// 16 warps: four per TMEM lane quadrant, each owning 32 of the 128 columns,
// so the epilogues (TMEM -> SiLU -> BF16 tile) run on 512 threads.
constexpr int kMlpThreads = 512;
constexpr int kColGroups = kMlpThreads / 128;      // column groups per row
constexpr int kColsPerThread = H / kColGroups;      // 32
// dynamic shared memory map (bytes)
constexpr int SM_W1 = 0, SM_W2 = SM_W1 + H * D * 2, SM_W3 = SM_W2 + H * H * 2, SM_X = SM_W3 + H * H * 2,
              SM_ACT = SM_X + TILE * D * 2, SM_W4 = SM_ACT + TILE * H * 2, SM_RED = SM_W4 + H * 4,
              SM_TOTAL = SM_RED + kColGroups * TILE * 4;
// TMEM columns
constexpr uint32_t TM_Z1 = 0, TM_Z2 = 128, TM_Z3 = 256, TM_T = 384;

// Forward epilogue of one hidden layer: each thread owns row q and
// kColsPerThread columns from c0 of z (TMEM at ta).  Writes h = SiLU(z) as
// the next BF16 operand tile (column 127 held at 1) and puts SiLU'(z) back
// into z's TMEM columns, where the gradient epilogue of this layer reads it,
// so the sigmoid is evaluated once per element.
__device__ __forceinline__ void epi_fwd(uint32_t ta, unsigned char* act, int q, int c0) {
#pragma unroll 1
    for (int cc = 0; cc < kColsPerThread; cc += 16) {
        float z[16], v[16], d[16];
        umma::tmem_ld16(ta + c0 + cc, z);
#pragma unroll
        for (int e = 0; e < 16; e++) {
            const float s = sigm(z[e]);
            v[e] = z[e] * s;
            d[e] = dsilu(z[e], s);
        }
        if (c0 + cc + 16 == H) v[15] = 1.f;
        umma::tmem_st16(ta + c0 + cc, d);
#pragma unroll
        for (int h8 = 0; h8 < 2; h8++) {
            uint4 o;
            o.x = umma::pack_bf16(v[8 * h8 + 0], v[8 * h8 + 1]);
            o.y = umma::pack_bf16(v[8 * h8 + 2], v[8 * h8 + 3]);
            o.z = umma::pack_bf16(v[8 * h8 + 4], v[8 * h8 + 5]);
            o.w = umma::pack_bf16(v[8 * h8 + 6], v[8 * h8 + 7]);
            *reinterpret_cast<uint4*>(act + umma::il_off(q, c0 + cc + 8 * h8, H)) = o;
        }
    }
    umma::tmem_wait_st();
}

// Gradient epilogue: g = t * SiLU'(z) from the t accumulator (ta) and the
// SiLU'(z) the forward epilogue left at td; column 127 held at 0.
__device__ __forceinline__ void epi_bwd(uint32_t ta, uint32_t td, unsigned char* act, int q, int c0) {
#pragma unroll 1
    for (int cc = 0; cc < kColsPerThread; cc += 16) {
        float v[16], d[16];
        umma::tmem_ld16(ta + c0 + cc, v);
        umma::tmem_ld16(td + c0 + cc, d);
#pragma unroll
        for (int e = 0; e < 16; e++) v[e] *= d[e];
        if (c0 + cc + 16 == H) v[15] = 0.f;
#pragma unroll
        for (int h8 = 0; h8 < 2; h8++) {
            uint4 o;
            o.x = umma::pack_bf16(v[8 * h8 + 0], v[8 * h8 + 1]);
            o.y = umma::pack_bf16(v[8 * h8 + 2], v[8 * h8 + 3]);
            o.z = umma::pack_bf16(v[8 * h8 + 4], v[8 * h8 + 5]);
            o.w = umma::pack_bf16(v[8 * h8 + 6], v[8 * h8 + 7]);
            *reinterpret_cast<uint4*>(act + umma::il_off(q, c0 + cc + 8 * h8, H)) = o;
        }
    }
}

__global__ void __launch_bounds__(kMlpThreads, 1)
k_sg_mlp(const uint16_t* __restrict__ img, const float* __restrict__ vec, const int* __restrict__ nrows,
         const uint16_t* __restrict__ X, float* __restrict__ bout, float* __restrict__ gxout, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tbase;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int q = 32 * (w & 3) + lane;          // tile row owned by this thread
    const int c0 = kColsPerThread * (w >> 2);   // first of its columns
    const int R = *nrows;
    const int ntiles = (R + TILE - 1) / TILE;
    if ((int)blockIdx.x >= ntiles) return;      // uniform per block; nothing allocated yet

    // weights (72 KB) and the output vector, once per CTA
    {
        const uint4* src = reinterpret_cast<const uint4*>(img);
        uint4* dst = reinterpret_cast<uint4*>(sm + SM_W1);
        for (int e = t; e < IMG_N * 2 / 16; e += kMlpThreads) dst[e] = src[e];
        float* w4 = reinterpret_cast<float*>(sm + SM_W4);
        for (int e = t; e < H; e += kMlpThreads) w4[e] = vec[V_W4 + e];
    }
    if (w == 0) {
        umma::tmem_alloc(&tbase, 512);
        umma::tmem_relinquish();
    }
    if (t == 0) umma::mbar_init(&mbar, 1);
    to_mma();
    const uint32_t tm = tbase;
    const uint32_t tl = tm + ((uint32_t)(32 * (w & 3)) << 16);   // this warp's TMEM lanes
    const uint32_t sW1 = umma::smem_u32(sm + SM_W1), sW2 = umma::smem_u32(sm + SM_W2),
                   sW3 = umma::smem_u32(sm + SM_W3), sX = umma::smem_u32(sm + SM_X),
                   sA = umma::smem_u32(sm + SM_ACT);
    unsigned char* act = sm + SM_ACT;
    const float* w4 = reinterpret_cast<const float*>(sm + SM_W4);
    float* red = reinterpret_cast<float*>(sm + SM_RED);
    const float b0 = vec[V_B0], bs = vec[V_BS];
    uint32_t ph = 0;
    bool ok = true;

    // The descriptor tile of the next 128 rows: 8 KB, one 16-byte piece per
    // thread, loaded into a register while the current tile is computed.
    static_assert(TILE * D * 2 / 16 == kMlpThreads, "one 16-byte piece of the descriptor tile per thread");
    uint4 xnext = reinterpret_cast<const uint4*>(X + (size_t)blockIdx.x * TILE * D)[t];

    // Wait for the MMAs of this step, then (after the epilogue) hand the new
    // operand tile to the issuing thread; a wait that ran out ends every
    // thread at the next hand-off.
#define SG_WAIT()                                                     \
    do {                                                              \
        if (ok) {                                                     \
            ok = umma::mbar_wait(&mbar, ph);                          \
            if (ok) ph ^= 1u;                                         \
        }                                                             \
        umma::fence_after();                                          \
    } while (0)
#define SG_HANDOFF()                                                  \
    do {                                                              \
        if (!to_mma_and(ok)) { ok = false; goto done; }               \
    } while (0)

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        reinterpret_cast<uint4*>(sm + SM_X)[t] = xnext;                // operand layout already
        SG_HANDOFF();
        if (t == 0) issue(tm + TM_Z1, sX, D, false, sW1, D, false, H, D / 16, &mbar);
        SG_WAIT();
        if (tile + (int)gridDim.x < ntiles)                           // X is free once z1 is done
            xnext = reinterpret_cast<const uint4*>(X + (size_t)(tile + gridDim.x) * TILE * D)[t];
        epi_fwd(tl + TM_Z1, act, q, c0);                              // h1, SiLU'(z1) -> TM_Z1
        SG_HANDOFF();
        if (t == 0) issue(tm + TM_Z2, sA, H, false, sW2, H, false, H, H / 16, &mbar);
        SG_WAIT();
        epi_fwd(tl + TM_Z2, act, q, c0);                              // h2, SiLU'(z2) -> TM_Z2
        SG_HANDOFF();
        if (t == 0) issue(tm + TM_Z3, sA, H, false, sW3, H, false, H, H / 16, &mbar);
        SG_WAIT();
        {   // output layer and g3 = bs * w4 * SiLU'(z3)
            float y = 0.f;
#pragma unroll 1
            for (int cc = 0; cc < kColsPerThread; cc += 16) {
                float z[16];
                umma::tmem_ld16(tl + TM_Z3 + c0 + cc, z);
                float g[16];
#pragma unroll
                for (int e = 0; e < 16; e++) {
                    const int col = c0 + cc + e;
                    const float s = sigm(z[e]);
                    const float hv = col == H - 1 ? 1.f : z[e] * s;
                    y += hv * w4[col];
                    g[e] = col == H - 1 ? 0.f : bs * w4[col] * dsilu(z[e], s);
                }
#pragma unroll
                for (int h8 = 0; h8 < 2; h8++) {
                    uint4 o;
                    o.x = umma::pack_bf16(g[8 * h8 + 0], g[8 * h8 + 1]);
                    o.y = umma::pack_bf16(g[8 * h8 + 2], g[8 * h8 + 3]);
                    o.z = umma::pack_bf16(g[8 * h8 + 4], g[8 * h8 + 5]);
                    o.w = umma::pack_bf16(g[8 * h8 + 6], g[8 * h8 + 7]);
                    *reinterpret_cast<uint4*>(act + umma::il_off(q, c0 + cc + 8 * h8, H)) = o;
                }
            }
            red[(w >> 2) * TILE + q] = y;
        }
        SG_HANDOFF();
        {
            const int row = tile * TILE + q;
            if (c0 == 0 && row < R) {
                float y = 0.f;
#pragma unroll
                for (int g = 0; g < kColGroups; g++) y += red[g * TILE + q];
                bout[row] = b0 + bs * y;
            }
        }
        if (t == 0) issue(tm + TM_T, sA, H, false, sW3, H, true, H, H / 16, &mbar);   // t2 = g3 W3^T
        SG_WAIT();
        epi_bwd(tl + TM_T, tl + TM_Z2, act, q, c0);                   // g2
        SG_HANDOFF();
        if (t == 0) issue(tm + TM_T, sA, H, false, sW2, H, true, H, H / 16, &mbar);   // t1 = g2 W2^T
        SG_WAIT();
        epi_bwd(tl + TM_T, tl + TM_Z1, act, q, c0);                   // g1
        SG_HANDOFF();
        if (t == 0) issue(tm + TM_T, sA, H, false, sW1, D, true, D, H / 16, &mbar);   // gx = g1 W1^T
        SG_WAIT();
        if ((w >> 2) < D / 16) {                // gx has D = 32 columns: two groups of 16
            const int row = tile * TILE + q;
            const int cg = 16 * (w >> 2);
            float v[16];
            umma::tmem_ld16(tl + TM_T + cg, v);
            if (row < R) {
                float4* dst = reinterpret_cast<float4*>(gxout + (size_t)row * D + cg);
#pragma unroll
                for (int e = 0; e < 4; e++) dst[e] = make_float4(v[4 * e], v[4 * e + 1], v[4 * e + 2], v[4 * e + 3]);
            }
        }
        umma::fence_before();
        // the next tile's first hand-off orders these TMEM reads before its MMAs
    }
done:
    if (!ok) {
        if (t == 0) atomicCAS(err + 1, 0, 1);
        // a thread whose own wait ran out still holds that phase: give the
        // MMA in flight a bounded chance to land before TMEM is released
        umma::mbar_wait(&mbar, ph);
    }
    umma::fence_before();
    __syncthreads();
    if (w == 0) umma::tmem_dealloc(tm, 512);
#undef SG_WAIT
#undef SG_HANDOFF
}

// ------------------------------------------------------------------ forces
__global__ void __launch_bounds__(256)
k_sg_force(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ cnt,
           const int* __restrict__ list, int cap, int na, const int* __restrict__ aoff,
           const int* __restrict__ row_i, const int* __restrict__ row_s, const int* __restrict__ partner,
           const float* __restrict__ b, const float* __restrict__ gx, const float* __restrict__ vec,
           double* __restrict__ F, double* __restrict__ part) {
    __shared__ double smr[32 * kNV];
    double h[9], hi[9];
    load_cell(hh, h, hi);
    double acc[kNV];
#pragma unroll
    for (int k = 0; k < kNV; k++) acc[k] = 0.0;
    const int R = aoff[na];
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
        const int i = row_i[r], j = list[(size_t)i * cap + row_s[r]];
        double dx, dy, dz;
        bond_vec(pos, i, j, h, hi, dx, dy, dz);
        const double rij = sqrt(norm2_rn(dx, dy, dz));
        const double fcut = sw_fc(rij), dfcut = sw_dfc(rij);
        const double e1 = exp(-BETA1_CC * rij), e2 = exp(-BETA2_CC * rij), e3 = exp(-BETA3_CC * rij);
        const double va = B1_CC * e1 + B2_CC * e2 + B3_CC * e3;
        if (i < j) {   // pair term once per bond (AI:325-365)
            const double ea = A_CC * exp(-ALPHA_CC * rij);
            const double vr = (1.0 + Q_CC / rij) * ea;
            const double dvr = (-Q_CC / (rij * rij)) * ea + (1.0 + Q_CC / rij) * (-ALPHA_CC) * ea;
            const double dva = -BETA1_CC * B1_CC * e1 - BETA2_CC * B2_CC * e2 - BETA3_CC * B3_CC * e3;
            const double bbar = 0.5 * ((double)b[r] + (double)b[partner[r]]);
            acc[0] += fcut * (vr - bbar * va);
            const double fpair = (dfcut * (vr - bbar * va) + fcut * (dvr - bbar * dva)) / rij;
            atomic_add3(F, i, fpair * dx, fpair * dy, fpair * dz);
            atomic_add3(F, j, -fpair * dx, -fpair * dy, -fpair * dz);
            const double d[3] = {dx, dy, dz};
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int c = 0; c < 3; c++) acc[1 + 3 * a + c] -= d[a] * fpair * d[c];
        }
        // three-body block of centre i (AI:368-390) with db_ij/dr_k from the network
        float gxr[D];
        const float4* gr = reinterpret_cast<const float4*>(gx + (size_t)r * D);
#pragma unroll
        for (int e = 0; e < D / 4; e++) {
            const float4 v = gr[e];
            gxr[4 * e] = v.x * vec[V_SINV + 4 * e];
            gxr[4 * e + 1] = v.y * vec[V_SINV + 4 * e + 1];
            gxr[4 * e + 2] = v.z * vec[V_SINV + 4 * e + 2];
            gxr[4 * e + 3] = v.w * vec[V_SINV + 4 * e + 3];
        }
        gxr[D - 1] = 0.f;
        const double coef = -0.5 * fcut * va;
        const double rinv = 1.0 / rij;
        const double ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;
        double fix = 0.0, fiy = 0.0, fiz = 0.0;
        for (int kn = 0; kn < cnt[i]; kn++) {
            const int k = list[(size_t)i * cap + kn];
            if (k == j) continue;
            double kx, ky, kz;
            bond_vec(pos, i, k, h, hi, kx, ky, kz);
            const double rk = sqrt(norm2_rn(kx, ky, kz));
            if (rk > DMAX_CC) continue;
            const double fk = sw_fc(rk);
            if (fk < 1e-15) continue;
            const double dfk = sw_dfc(rk);
            const double ct = clamp1((dx * kx + dy * ky + dz * kz) / (rij * rk));
            float Tr[NR], dTr[NR], Ta[NA], dTa[NA];
            cheb<NR>((float)((rk - RHO_C) / RHO_W), Tr, dTr);
            cheb<NA>((float)ct, Ta, dTa);
            float A1 = 0.f, A2 = 0.f;
#pragma unroll
            for (int a = 0; a < NR; a++) {
                const float phi = (float)fk * Tr[a];
                const float dphi = (float)dfk * Tr[a] + (float)fk * dTr[a] * (float)(1.0 / RHO_W);
                float s1 = 0.f, s2 = 0.f;
#pragma unroll
                for (int bb = 0; bb < NA; bb++) {
                    s1 += gxr[a * NA + bb] * Ta[bb];
                    s2 += gxr[a * NA + bb] * dTa[bb];
                }
                A1 += dphi * s1;
                A2 += phi * s2;
            }
            const double rki = 1.0 / rk;
            const double rx = kx * rki, ry = ky * rki, rz = kz * rki;
            const double fx = coef * ((double)A1 * rx + (double)A2 * (ux - ct * rx) * rki);
            const double fy = coef * ((double)A1 * ry + (double)A2 * (uy - ct * ry) * rki);
            const double fz = coef * ((double)A1 * rz + (double)A2 * (uz - ct * rz) * rki);
            atomic_add3(F, k, fx, fy, fz);
            fix -= fx; fiy -= fy; fiz -= fz;
        }
        if (fix != 0.0 || fiy != 0.0 || fiz != 0.0) atomic_add3(F, i, fix, fiy, fiz);
    }
    block_sum_store<kNV>(acc, smr, part + (size_t)blockIdx.x * kNV);
}

__global__ void k_sg_pack(const double* __restrict__ P, uint16_t* __restrict__ img, float* __restrict__ vec) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < IMG_N; e += gridDim.x * blockDim.x) {
        double v;
        uint32_t off;
        if (e < IMG_W2) {                                   // W1 image: row h, column d
            const int hrow = e / D, d = e % D;
            v = P[OW1 + d * H + hrow];
            off = umma::il_off(hrow, d, D);
            reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<unsigned char*>(img) + IMG_W1 * 2 + off)[0] =
                __float2bfloat16_rn((float)v);
        } else {
            const int l = e < IMG_W3 ? 2 : 3;
            const int ee = e - (l == 2 ? IMG_W2 : IMG_W3);
            const int o = ee / H, k = ee % H;               // row = output unit, column = input unit
            v = P[(l == 2 ? OW2 : OW3) + k * H + o];
            off = umma::il_off(o, k, H);
            reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<unsigned char*>(img) + (l == 2 ? IMG_W2 : IMG_W3) * 2 +
                                             off)[0] = __float2bfloat16_rn((float)v);
        }
    }
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < V_N; e += gridDim.x * blockDim.x) {
        float v;
        if (e < V_M) v = (float)P[OW4 + e];
        else if (e < V_SINV) v = (float)P[OM + (e - V_M)];
        else if (e < V_B0) v = (float)(1.0 / P[OS + (e - V_SINV)]);
        else if (e == V_B0) v = (float)P[OB0];
        else v = (float)P[OBS];
        vec[e] = v;
    }
}

}  // namespace

cudaError_t work_alloc(Work& w, int na, int cap) {
    if (na <= w.na_cap && cap == w.cap) return cudaSuccess;
    work_free(w);
    const int rcap = ((na * cap + TILE - 1) / TILE) * TILE;
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    };
    A((void**)&w.acnt, sizeof(int) * (size_t)na);
    A((void**)&w.aoff, sizeof(int) * ((size_t)na + 1));
    A((void**)&w.row_i, sizeof(int) * (size_t)rcap);
    A((void**)&w.row_s, sizeof(int) * (size_t)rcap);
    A((void**)&w.rowid, sizeof(int) * (size_t)na * cap);
    A((void**)&w.partner, sizeof(int) * (size_t)rcap);
    A((void**)&w.X, sizeof(uint16_t) * (size_t)rcap * D);
    A((void**)&w.b, sizeof(float) * (size_t)rcap);
    A((void**)&w.gx, sizeof(float) * (size_t)rcap * D);
    A((void**)&w.part, sizeof(double) * (size_t)kRowBlocks * kNV);
    A((void**)&w.err, sizeof(int) * 4);
    A((void**)&w.bsum, sizeof(int) * ((size_t)na / 256 + 2));
    A((void**)&w.boff, sizeof(int) * ((size_t)na / 256 + 3));
    if (e == cudaSuccess) e = cudaMemset(w.err, 0, sizeof(int) * 4);
    if (e != cudaSuccess) {
        work_free(w);
        return e;
    }
    w.na_cap = na;
    w.r_cap = rcap;
    w.cap = cap;
    return cudaSuccess;
}

void work_free(Work& w) {
    cudaFree(w.acnt); cudaFree(w.aoff); cudaFree(w.row_i); cudaFree(w.row_s); cudaFree(w.rowid);
    cudaFree(w.partner); cudaFree(w.X); cudaFree(w.b); cudaFree(w.gx); cudaFree(w.part); cudaFree(w.err);
    cudaFree(w.bsum); cudaFree(w.boff);
    w = Work{};
}

cudaError_t pack_params(const double* P, uint16_t* img, float* vec, cudaStream_t st) {
    k_sg_pack<<<64, 256, 0, st>>>(P, img, vec);
    return cudaGetLastError();
}

cudaError_t build_rows(Work& w, const float* vec, const double* pos, const double* hh, const int* cnt,
                       const int* list, int cap, int na, cudaStream_t st, const int* gate) {
    if (na > w.na_cap || cap != w.cap) return cudaErrorInvalidValue;
    w.na_used = na;
    const int nb = (na + kScanBlock - 1) / kScanBlock;
    k_sg_count<<<nb, kScanBlock, 0, st>>>(pos, hh, cnt, list, cap, na, w.acnt, gate, w.aoff, w.bsum);
    k_sg_scan<<<1, 1024, 0, st>>>(w.bsum, nb, w.boff);
    k_sg_rows<<<nb, kScanBlock, 0, st>>>(pos, hh, cnt, list, cap, na, w.aoff, w.row_i, w.row_s, w.rowid, gate, w.boff);
    k_sg_desc<<<kRowBlocks, 128, 0, st>>>(pos, hh, cnt, list, cap, na, w.aoff, w.row_i, w.row_s, w.rowid, vec,
                                          w.r_cap, w.X, w.partner, w.err);
    return cudaGetLastError();
}

cudaError_t run_mlp(Work& w, const uint16_t* img, const float* vec, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_sg_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize, SM_TOTAL);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    // the row count stays on the device (aoff[na] of the last build)
    k_sg_mlp<<<kSMs, kMlpThreads, SM_TOTAL, st>>>(img, vec, w.aoff + w.na_used, w.X, w.b, w.gx, w.err);
    return cudaGetLastError();
}

cudaError_t assemble(Work& w, const float* vec, const double* pos, const double* hh, const int* cnt,
                     const int* list, int cap, int na, double* F, double* part, cudaStream_t st) {
    k_sg_force<<<kRowBlocks, 256, 0, st>>>(pos, hh, cnt, list, cap, na, w.aoff, w.row_i, w.row_s, w.partner, w.b,
                                           w.gx, vec, F, part);
    return cudaGetLastError();
}

cudaError_t rebo_forces(Work& w, const uint16_t* img, const float* vec, const double* pos, const double* hh,
                        const int* cnt, const int* list, int cap, int na, double* F, double* part,
                        cudaStream_t st, const int* gate) {
    cudaError_t e = build_rows(w, vec, pos, hh, cnt, list, cap, na, st, gate);
    if (e == cudaSuccess) e = run_mlp(w, img, vec, st);
    if (e == cudaSuccess) e = assemble(w, vec, pos, hh, cnt, list, cap, na, F, part, st);
    return e;
}

}  // namespace sg
}  // namespace fmd
