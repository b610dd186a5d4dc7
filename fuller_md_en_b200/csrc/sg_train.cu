// sg_train.cu -- training of the learned bond-order potential on the GPU.
//
// One step on a snapshot with reference REBO energy, forces and virial:
//   inference path (surrogate.cu)            b, db/dx, E, F, W
//   k_sg_lambda                              dL/dF per atom, sum dF^2
//   k_sg_adjoint                             per row dL/db and dL/d(db/dx)
//   k_sg_chain  (tcgen05, 10 GEMMs / tile)   double backpropagation through
//                                            the network; writes the BF16
//                                            operand tiles of the weight
//                                            gradients, sums dL/dw4
//   k_sg_wgrad  (tcgen05)                    dW_l = sum over rows, reduced in
//                                            TMEM per CTA
//   k_sg_adam                                FP64 master weights, then repack
// The loss is  wF mean(dF^2) + wE (dE/na)^2 + wW mean((dW/na)^2)  with dF over
// the REBO forces; every step restates oracle/sg_oracle.py:mlp_backward with
// the same BF16 rounding points.
#include <cuda_bf16.h>

#include "kernels.h"
#include "sg_dev.cuh"
#include "sg_train.cuh"
#include "umma.cuh"

namespace fmd {
namespace sg {
namespace {

using namespace dev;

// ------------------------------------------------------------- adjoints
__global__ void __launch_bounds__(256)
k_sg_lambda(const double* __restrict__ F, const double* __restrict__ Fref, int na, double wF,
            double* __restrict__ lamF, double* __restrict__ part) {
    __shared__ double sm[32];
    double acc[1] = {0.0};
    const double k = 2.0 * wF / (3.0 * na);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 3 * na; e += gridDim.x * blockDim.x) {
        const double d = F[e] - Fref[e];
        lamF[e] = k * d;
        acc[0] += d * d;
    }
    block_sum_store<1>(acc, sm, part + blockIdx.x);
}

// sc: {E, W9} of the prediction; ref: {E, W9} of the reference.
__global__ void k_sg_loss(const double* __restrict__ sc, const double* __restrict__ ref,
                          const double* __restrict__ sumdf2, int na, double wE, double wF, double wW,
                          double* __restrict__ lam, double* __restrict__ loss_acc) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double n2 = (double)na * na;
    const double dE = sc[0] - ref[0];
    double lw = 0.0;
    lam[0] = 2.0 * wE * dE / n2;
    for (int a = 0; a < 9; a++) {
        const double dW = sc[1 + a] - ref[1 + a];
        lam[1 + a] = 2.0 * wW * dW / (9.0 * n2);
        lw += dW * dW;
    }
    loss_acc[0] += wF * sumdf2[0] / (3.0 * na) + wE * dE * dE / n2 + wW * lw / (9.0 * n2);
    loss_acc[1] += sumdf2[0] / (3.0 * na);          // mean dF^2 (for the force RMSE)
}

// One thread per row: beta = dL/db, and the U tile row = dL/d(db/dxn).
__global__ void __launch_bounds__(128)
k_sg_adjoint(const double* __restrict__ pos, const double* __restrict__ hh, const int* __restrict__ cnt,
             const int* __restrict__ list, int cap, int na, const int* __restrict__ aoff,
             const int* __restrict__ row_i, const int* __restrict__ row_s, const float* __restrict__ vec,
             const double* __restrict__ lamF, const double* __restrict__ lam, int r_cap,
             float* __restrict__ beta, uint16_t* __restrict__ U) {
    double h[9], hi[9];
    load_cell(hh, h, hi);
    const int R = aoff[na];
    const int Rpad = (R + TILE - 1) / TILE * TILE;
    const double lE = lam[0];
    double LW[9];
#pragma unroll
    for (int a = 0; a < 9; a++) LW[a] = lam[1 + a];
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < Rpad && r < r_cap; r += gridDim.x * blockDim.x) {
        float u[D];
#pragma unroll
        for (int f = 0; f < D; f++) u[f] = 0.f;
        float bt = 0.f;
        if (r < R) {
            const int i = row_i[r], j = list[(size_t)i * cap + row_s[r]];
            double dx, dy, dz;
            bond_vec(pos, i, j, h, hi, dx, dy, dz);
            const double rij = sqrt(norm2_rn(dx, dy, dz));
            const double fcut = sw_fc(rij), dfcut = sw_dfc(rij);
            const double e1 = exp(-BETA1_CC * rij), e2 = exp(-BETA2_CC * rij), e3 = exp(-BETA3_CC * rij);
            const double va = B1_CC * e1 + B2_CC * e2 + B3_CC * e3;
            const double dva = -BETA1_CC * B1_CC * e1 - BETA2_CC * B2_CC * e2 - BETA3_CC * B3_CC * e3;
            // dL/dfpair through F_i, F_j (pair force) and W (pair virial)
            const double d[3] = {dx, dy, dz};
            double dfp = 0.0, dWd = 0.0;
#pragma unroll
            for (int a = 0; a < 3; a++) {
                dfp += (lamF[3 * i + a] - lamF[3 * j + a]) * d[a];
#pragma unroll
                for (int c = 0; c < 3; c++) dWd += d[a] * LW[3 * a + c] * d[c];
            }
            dfp -= dWd;
            const double phi = -(dfcut * va + fcut * dva) / rij;     // d fpair / d b_bar
            bt = (float)(-0.5 * fcut * va * lE + 0.5 * phi * dfp);
            // dL/d(db/dxn): three-body forces F_k += w db/dr_k, F_i -= the same
            const double w = -0.5 * fcut * va;
            const double rinv = 1.0 / rij;
            const double ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;
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
                const double rki = 1.0 / rk;
                const double rx = kx * rki, ry = ky * rki, rz = kz * rki;
                const double lx = lamF[3 * k] - lamF[3 * i], ly = lamF[3 * k + 1] - lamF[3 * i + 1],
                             lz = lamF[3 * k + 2] - lamF[3 * i + 2];
                const float p1 = (float)(w * (lx * rx + ly * ry + lz * rz));                 // w dl . rhat_k
                const float p2 = (float)(w * (lx * (ux - ct * rx) + ly * (uy - ct * ry) + lz * (uz - ct * rz)) * rki);
                float Tr[NR], dTr[NR], Ta[NA], dTa[NA];
                cheb<NR>((float)((rk - RHO_C) / RHO_W), Tr, dTr);
                cheb<NA>((float)ct, Ta, dTa);
#pragma unroll
                for (int a = 0; a < NR; a++) {
                    const float phi_a = (float)fk * Tr[a];
                    const float dphi_a = (float)dfk * Tr[a] + (float)fk * dTr[a] * (float)(1.0 / RHO_W);
#pragma unroll
                    for (int b = 0; b < NA; b++) u[a * NA + b] += dphi_a * Ta[b] * p1 + phi_a * dTa[b] * p2;
                }
            }
#pragma unroll
            for (int f = 0; f < D - 1; f++) u[f] *= vec[V_SINV + f];
            u[D - 1] = 0.f;
        }
        beta[r] = bt;
        unsigned char* tile = reinterpret_cast<unsigned char*>(U) + (size_t)(r / TILE) * TILE * D * 2;
        const int q = r % TILE;
#pragma unroll
        for (int c8 = 0; c8 < D / 8; c8++) {
            uint4 v;
            v.x = umma::pack_bf16(u[8 * c8 + 0], u[8 * c8 + 1]);
            v.y = umma::pack_bf16(u[8 * c8 + 2], u[8 * c8 + 3]);
            v.z = umma::pack_bf16(u[8 * c8 + 4], u[8 * c8 + 5]);
            v.w = umma::pack_bf16(u[8 * c8 + 6], u[8 * c8 + 7]);
            *reinterpret_cast<uint4*>(tile + umma::il_off(q, 8 * c8, D)) = v;
        }
    }
}

// ------------------------------------------------------------- chain
constexpr int kThreads = 256;
constexpr int C_W1 = 0, C_W2 = C_W1 + H * D * 2, C_W3 = C_W2 + H * H * 2, C_X = C_W3 + H * H * 2,
              C_U = C_X + TILE * D * 2, C_ACT = C_U + TILE * D * 2, C_E1 = C_ACT + TILE * H * 2,
              C_E2 = C_E1 + TILE * H * 2, C_W4 = C_E2 + TILE * H * 2, C_DW4 = C_W4 + H * 4,
              C_BETA = C_DW4 + H * 4, C_TOTAL = C_BETA + TILE * 4;
constexpr uint32_t T_Z1 = 0, T_Z2 = 128, T_Z3 = 256, T_T = 384;

// Sums 16 column values over the 32 rows of this warp and adds them to acc.
__device__ __forceinline__ void colsum16(const float* v, float* acc, int col, int lane) {
#pragma unroll
    for (int e = 0; e < 16; e++) {
        float x = v[e];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) atomicAdd(&acc[col + e], x);
    }
}

__device__ __forceinline__ unsigned char* gtile(uint16_t* buf, int tile) {
    return reinterpret_cast<unsigned char*>(buf) + (size_t)tile * TILE * H * 2;
}

__global__ void __launch_bounds__(kThreads, 1)
k_sg_chain(const uint16_t* __restrict__ img, const float* __restrict__ vec, const int* __restrict__ nrows,
           const uint16_t* __restrict__ X, const uint16_t* __restrict__ Ut, const float* __restrict__ beta,
           OperandTiles out, float* __restrict__ dw4_glob, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tbase;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int q = 32 * (w & 3) + lane;
    const int c0 = 64 * (w >> 2);
    const int R = *nrows;
    const int ntiles = (R + TILE - 1) / TILE;
    if ((int)blockIdx.x >= ntiles) return;
    {
        const uint4* src = reinterpret_cast<const uint4*>(img);
        uint4* dst = reinterpret_cast<uint4*>(sm + C_W1);
        for (int e = t; e < IMG_N * 2 / 16; e += kThreads) dst[e] = src[e];
        float* w4 = reinterpret_cast<float*>(sm + C_W4);
        float* dw4 = reinterpret_cast<float*>(sm + C_DW4);
        for (int e = t; e < H; e += kThreads) { w4[e] = vec[V_W4 + e]; dw4[e] = 0.f; }
    }
    if (w == 0) {
        umma::tmem_alloc(&tbase, 512);
        umma::tmem_relinquish();
    }
    if (t == 0) umma::mbar_init(&mbar, 1);
    to_mma();
    const uint32_t tm = tbase;
    const uint32_t tl = tm + ((uint32_t)(32 * (w & 3)) << 16);
    const uint32_t sW1 = umma::smem_u32(sm + C_W1), sW2 = umma::smem_u32(sm + C_W2), sW3 = umma::smem_u32(sm + C_W3),
                   sX = umma::smem_u32(sm + C_X), sU = umma::smem_u32(sm + C_U), sA = umma::smem_u32(sm + C_ACT);
    unsigned char* act = sm + C_ACT;
    unsigned char* E1 = sm + C_E1;
    unsigned char* E2 = sm + C_E2;
    const float* w4 = reinterpret_cast<const float*>(sm + C_W4);
    float* dw4 = reinterpret_cast<float*>(sm + C_DW4);
    float* sbeta = reinterpret_cast<float*>(sm + C_BETA);
    const float bs = vec[V_BS];
    uint32_t ph = 0;
    bool ok = true;

#define SG_WAIT()                                                     \
    do {                                                              \
        const bool _w = umma::mbar_wait(&mbar, ph);                   \
        ph ^= 1u;                                                     \
        umma::fence_after();                                          \
        if (!__syncthreads_and(_w)) { ok = false; goto done; }        \
    } while (0)

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        {
            const uint4* sx = reinterpret_cast<const uint4*>(X + (size_t)tile * TILE * D);
            const uint4* su = reinterpret_cast<const uint4*>(Ut + (size_t)tile * TILE * D);
            uint4* dx = reinterpret_cast<uint4*>(sm + C_X);
            uint4* du = reinterpret_cast<uint4*>(sm + C_U);
            for (int e = t; e < TILE * D * 2 / 16; e += kThreads) { dx[e] = sx[e]; du[e] = su[e]; }
            if (t < TILE) sbeta[t] = beta[(size_t)tile * TILE + t];
        }
        to_mma();
        const float ybar = sbeta[q] * bs;
        // ---- forward
        if (t == 0) issue(tm + T_Z1, sX, D, false, sW1, D, false, H, D / 16, &mbar);
        SG_WAIT();
        for (int cc = 0; cc < 64; cc += 16) {
            float z[16], v[16];
            umma::tmem_ld16(tl + T_Z1 + c0 + cc, z);
            for (int e = 0; e < 16; e++) v[e] = (c0 + cc + e == H - 1) ? 1.f : z[e] * sigm(z[e]);
            st_tile16(act, q, c0 + cc, v);
            st_tile16(gtile(out.h1, tile), q, c0 + cc, v);
        }
        to_mma();
        if (t == 0) issue(tm + T_Z2, sA, H, false, sW2, H, false, H, H / 16, &mbar);
        SG_WAIT();
        for (int cc = 0; cc < 64; cc += 16) {
            float z[16], v[16];
            umma::tmem_ld16(tl + T_Z2 + c0 + cc, z);
            for (int e = 0; e < 16; e++) v[e] = (c0 + cc + e == H - 1) ? 1.f : z[e] * sigm(z[e]);
            st_tile16(act, q, c0 + cc, v);
            st_tile16(gtile(out.h2, tile), q, c0 + cc, v);
        }
        to_mma();
        if (t == 0) issue(tm + T_Z3, sA, H, false, sW3, H, false, H, H / 16, &mbar);
        SG_WAIT();
        for (int cc = 0; cc < 64; cc += 16) {   // g3 = bs w4 SiLU'(z3); dw4 += ybar h3
            float z[16], g[16], yh[16];
            umma::tmem_ld16(tl + T_Z3 + c0 + cc, z);
            for (int e = 0; e < 16; e++) {
                const int col = c0 + cc + e;
                const float s = sigm(z[e]);
                g[e] = col == H - 1 ? 0.f : bs * w4[col] * dsilu(z[e], s);
                yh[e] = ybar * (col == H - 1 ? 1.f : z[e] * s);
            }
            st_tile16(act, q, c0 + cc, g);
            st_tile16(gtile(out.g3, tile), q, c0 + cc, g);
            colsum16(yh, dw4, c0 + cc, lane);
        }
        // ---- gradient network
        to_mma();
        if (t == 0) issue(tm + T_T, sA, H, false, sW3, H, true, H, H / 16, &mbar);        // t2 = g3 W3^T
        SG_WAIT();
        for (int cc = 0; cc < 64; cc += 16) {
            float tv[16], z[16], g[16], e2[16];
            umma::tmem_ld16(tl + T_T + c0 + cc, tv);
            umma::tmem_ld16(tl + T_Z2 + c0 + cc, z);
            for (int e = 0; e < 16; e++) {
                const bool last = c0 + cc + e == H - 1;
                const float s = sigm(z[e]);
                g[e] = last ? 0.f : tv[e] * dsilu(z[e], s);
                e2[e] = last ? 0.f : tv[e] * d2silu(z[e], s);
            }
            st_tile16(act, q, c0 + cc, g);
            st_tile16(gtile(out.g2, tile), q, c0 + cc, g);
            st_tile16(E2, q, c0 + cc, e2);
        }
        to_mma();
        if (t == 0) issue(tm + T_T, sA, H, false, sW2, H, true, H, H / 16, &mbar);        // t1 = g2 W2^T
        SG_WAIT();
        for (int cc = 0; cc < 64; cc += 16) {
            float tv[16], z[16], g[16], e1[16];
            umma::tmem_ld16(tl + T_T + c0 + cc, tv);
            umma::tmem_ld16(tl + T_Z1 + c0 + cc, z);
            for (int e = 0; e < 16; e++) {
                const bool last = c0 + cc + e == H - 1;
                const float s = sigm(z[e]);
                g[e] = last ? 0.f : tv[e] * dsilu(z[e], s);
                e1[e] = last ? 0.f : tv[e] * d2silu(z[e], s);
            }
            st_tile16(gtile(out.g1, tile), q, c0 + cc, g);
            st_tile16(E1, q, c0 + cc, e1);
        }
        // ---- adjoint of the gradient network
        to_mma();
        if (t == 0) issue(tm + T_T, sU, D, false, sW1, D, false, H, D / 16, &mbar);        // gb1 = u W1
        SG_WAIT();
        for (int cc = 0; cc < 64; cc += 16) {
            float gb[16], z[16], e1[16], tb[16];
            umma::tmem_ld16(tl + T_T + c0 + cc, gb);
            umma::tmem_ld16(tl + T_Z1 + c0 + cc, z);
            ld_tile16(E1, q, c0 + cc, e1);
            for (int e = 0; e < 16; e++) {
                const bool last = c0 + cc + e == H - 1;
                tb[e] = last ? 0.f : gb[e] * dsilu(z[e], sigm(z[e]));
                e1[e] = last ? 0.f : gb[e] * e1[e];                                       // zd1
            }
            st_tile16(act, q, c0 + cc, tb);
            st_tile16(gtile(out.tb1, tile), q, c0 + cc, tb);
            st_tile16(E1, q, c0 + cc, e1);
        }
        to_mma();
        if (t == 0) issue(tm + T_T, sA, H, false, sW2, H, false, H, H / 16, &mbar);       // gb2 = tb1 W2
        SG_WAIT();
        for (int cc = 0; cc < 64; cc += 16) {
            float gb[16], z[16], e2[16], tb[16];
            umma::tmem_ld16(tl + T_T + c0 + cc, gb);
            umma::tmem_ld16(tl + T_Z2 + c0 + cc, z);
            ld_tile16(E2, q, c0 + cc, e2);
            for (int e = 0; e < 16; e++) {
                const bool last = c0 + cc + e == H - 1;
                tb[e] = last ? 0.f : gb[e] * dsilu(z[e], sigm(z[e]));
                e2[e] = last ? 0.f : gb[e] * e2[e];                                       // zd2
            }
            st_tile16(act, q, c0 + cc, tb);
            st_tile16(gtile(out.tb2, tile), q, c0 + cc, tb);
            st_tile16(E2, q, c0 + cc, e2);
        }
        to_mma();
        if (t == 0) issue(tm + T_T, sA, H, false, sW3, H, false, H, H / 16, &mbar);       // gb3 = tb2 W3
        SG_WAIT();
        for (int cc = 0; cc < 64; cc += 16) {   // dw4 += bs gb3 SiLU'(z3); zb3
            float gb[16], z[16], zb[16], dv[16];
            umma::tmem_ld16(tl + T_T + c0 + cc, gb);
            umma::tmem_ld16(tl + T_Z3 + c0 + cc, z);
            for (int e = 0; e < 16; e++) {
                const int col = c0 + cc + e;
                const bool last = col == H - 1;
                const float s = sigm(z[e]);
                dv[e] = last ? 0.f : bs * gb[e] * dsilu(z[e], s);
                zb[e] = last ? 0.f : gb[e] * bs * w4[col] * d2silu(z[e], s) + ybar * w4[col] * dsilu(z[e], s);
            }
            colsum16(dv, dw4, c0 + cc, lane);
            st_tile16(act, q, c0 + cc, zb);
            st_tile16(gtile(out.z3, tile), q, c0 + cc, zb);
        }
        // ---- adjoint of the forward network
        to_mma();
        if (t == 0) issue(tm + T_T, sA, H, false, sW3, H, true, H, H / 16, &mbar);        // hb2 = zb3 W3^T
        SG_WAIT();
        for (int cc = 0; cc < 64; cc += 16) {
            float hb[16], z[16], zd[16];
            umma::tmem_ld16(tl + T_T + c0 + cc, hb);
            umma::tmem_ld16(tl + T_Z2 + c0 + cc, z);
            ld_tile16(E2, q, c0 + cc, zd);
            for (int e = 0; e < 16; e++)
                zd[e] = (c0 + cc + e == H - 1) ? 0.f : zd[e] + hb[e] * dsilu(z[e], sigm(z[e]));
            st_tile16(act, q, c0 + cc, zd);
            st_tile16(gtile(out.z2, tile), q, c0 + cc, zd);
        }
        to_mma();
        if (t == 0) issue(tm + T_T, sA, H, false, sW2, H, true, H, H / 16, &mbar);        // hb1 = zb2 W2^T
        SG_WAIT();
        for (int cc = 0; cc < 64; cc += 16) {
            float hb[16], z[16], zd[16];
            umma::tmem_ld16(tl + T_T + c0 + cc, hb);
            umma::tmem_ld16(tl + T_Z1 + c0 + cc, z);
            ld_tile16(E1, q, c0 + cc, zd);
            for (int e = 0; e < 16; e++)
                zd[e] = (c0 + cc + e == H - 1) ? 0.f : zd[e] + hb[e] * dsilu(z[e], sigm(z[e]));
            st_tile16(gtile(out.z1, tile), q, c0 + cc, zd);
        }
        umma::fence_before();
        __syncthreads();
        umma::fence_after();
    }
done:
    if (!ok) {
        if (t == 0) atomicCAS(err + 2, 0, 1);
        umma::mbar_wait(&mbar, ph);
    }
    umma::fence_before();
    __syncthreads();
    if (ok)
        for (int e = t; e < H; e += kThreads) atomicAdd(&dw4_glob[e], dw4[e]);
    if (w == 0) umma::tmem_dealloc(tm, 512);
#undef SG_WAIT
}

// ------------------------------------------------------------- weight gradients
constexpr int G_A = 0, G_B = 32768, G_C = 65536, G_D = 98304, G_TOTAL = 131072;
constexpr uint32_t T_D1 = 0, T_D2 = 128, T_D3 = 256;

__device__ __forceinline__ void load_tile(unsigned char* dst, const unsigned char* src, int bytes, int t) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(dst);
    for (int e = t; e < bytes / 16; e += kThreads) d[e] = s[e];
}

__global__ void __launch_bounds__(kThreads, 1)
k_sg_wgrad(const int* __restrict__ nrows, const uint16_t* __restrict__ X, const uint16_t* __restrict__ Ut,
           OperandTiles in, float* __restrict__ grad, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tbase;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int R = *nrows;
    const int ntiles = (R + TILE - 1) / TILE;
    if ((int)blockIdx.x >= ntiles) return;
    if (w == 0) {
        umma::tmem_alloc(&tbase, 512);
        umma::tmem_relinquish();
    }
    if (t == 0) umma::mbar_init(&mbar, 1);
    to_mma();
    const uint32_t tm = tbase;
    const uint32_t sa = umma::smem_u32(sm + G_A), sb = umma::smem_u32(sm + G_B), sc = umma::smem_u32(sm + G_C),
                   sd = umma::smem_u32(sm + G_D);
    uint32_t ph = 0;
    bool ok = true;
    bool first = true;
    const uint32_t id1 = umma::idesc_bf16(128, D, true, true), id2 = umma::idesc_bf16(128, H, true, true);

#define SG_WAIT()                                                     \
    do {                                                              \
        const bool _w = umma::mbar_wait(&mbar, ph);                   \
        ph ^= 1u;                                                     \
        umma::fence_after();                                          \
        if (!__syncthreads_and(_w)) { ok = false; goto done; }        \
    } while (0)

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const size_t toff = (size_t)tile * TILE * H * 2, xoff = (size_t)tile * TILE * D * 2;
        // dW1^T += zb1^T x + g1^T u   (M = 128 hidden, N = 32 inputs, K = rows)
        load_tile(sm + G_A, reinterpret_cast<const unsigned char*>(in.z1) + toff, TILE * H * 2, t);
        load_tile(sm + G_B, reinterpret_cast<const unsigned char*>(X) + xoff, TILE * D * 2, t);
        load_tile(sm + G_C, reinterpret_cast<const unsigned char*>(in.g1) + toff, TILE * H * 2, t);
        load_tile(sm + G_D, reinterpret_cast<const unsigned char*>(Ut) + xoff, TILE * D * 2, t);
        to_mma();
        if (t == 0) {
            for (int s = 0; s < TILE / 16; s++)
                umma::mma_bf16(tm + T_D1, umma::desc_mn(sa, H, s), umma::desc_mn(sb, D, s), id1, !(first && s == 0));
            for (int s = 0; s < TILE / 16; s++)
                umma::mma_bf16(tm + T_D1, umma::desc_mn(sc, H, s), umma::desc_mn(sd, D, s), id1, 1);
            umma::commit(&mbar);
        }
        SG_WAIT();
        // dW2^T += zb2^T h1 + g2^T tb1 ; dW3^T += zb3^T h2 + g3^T tb2
        for (int l = 0; l < 2; l++) {
            const uint16_t* A1 = l == 0 ? in.z2 : in.z3;
            const uint16_t* B1 = l == 0 ? in.h1 : in.h2;
            const uint16_t* A2 = l == 0 ? in.g2 : in.g3;
            const uint16_t* B2 = l == 0 ? in.tb1 : in.tb2;
            load_tile(sm + G_A, reinterpret_cast<const unsigned char*>(A1) + toff, TILE * H * 2, t);
            load_tile(sm + G_B, reinterpret_cast<const unsigned char*>(B1) + toff, TILE * H * 2, t);
            load_tile(sm + G_C, reinterpret_cast<const unsigned char*>(A2) + toff, TILE * H * 2, t);
            load_tile(sm + G_D, reinterpret_cast<const unsigned char*>(B2) + toff, TILE * H * 2, t);
            to_mma();
            if (t == 0) {
                const uint32_t dcol = tm + (l == 0 ? T_D2 : T_D3);
                for (int s = 0; s < TILE / 16; s++)
                    umma::mma_bf16(dcol, umma::desc_mn(sa, H, s), umma::desc_mn(sb, H, s), id2, !(first && s == 0));
                for (int s = 0; s < TILE / 16; s++)
                    umma::mma_bf16(dcol, umma::desc_mn(sc, H, s), umma::desc_mn(sd, H, s), id2, 1);
                umma::commit(&mbar);
            }
            SG_WAIT();
        }
        first = false;
    }
    {   // this CTA's sums -> global (row = output unit, columns = input unit)
        const uint32_t tl = tm + ((uint32_t)(32 * (w & 3)) << 16);
        const int row = 32 * (w & 3) + lane;
        if (w < 4) {
            for (int c = 0; c < D; c += 16) {
                float v[16];
                umma::tmem_ld16(tl + T_D1 + c, v);
                for (int e = 0; e < 16; e++) atomicAdd(&grad[row * D + c + e], v[e]);
            }
        }
        const int half = 64 * (w >> 2);
        for (int l = 0; l < 2; l++) {
            float* G = grad + H * D + l * H * H;
            for (int c = half; c < half + 64; c += 16) {
                float v[16];
                umma::tmem_ld16(tl + (l == 0 ? T_D2 : T_D3) + c, v);
                for (int e = 0; e < 16; e++) atomicAdd(&G[row * H + c + e], v[e]);
            }
        }
    }
done:
    if (!ok) {
        if (t == 0) atomicCAS(err + 3, 0, 1);
        umma::mbar_wait(&mbar, ph);
    }
    umma::fence_before();
    __syncthreads();
    if (w == 0) umma::tmem_dealloc(tm, 512);
#undef SG_WAIT
}

// Gradient in the master layout (W[in][out]); only the network weights train.
__device__ __forceinline__ double grad_of(const float* g, int p) {
    if (p < OW2) {
        const int d = p / H, h = p % H;
        return g[h * D + d];
    }
    if (p < OW4) {
        const int l = p < OW3 ? 0 : 1;
        const int e = p - (l == 0 ? OW2 : OW3);
        const int k = e / H, o = e % H;
        return g[H * D + l * H * H + o * H + k];
    }
    return g[H * D + 2 * H * H + (p - OW4)];
}

__global__ void k_sg_adam(double* __restrict__ P, double* __restrict__ m, double* __restrict__ v,
                          const float* __restrict__ g, AdamArgs a) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < OM; p += gridDim.x * blockDim.x) {
        double gr = grad_of(g, p) * a.scale;
        if (a.clip > 0.0) gr = fmin(fmax(gr, -a.clip), a.clip);
        const double mm = a.b1 * m[p] + (1.0 - a.b1) * gr;
        const double vv = a.b2 * v[p] + (1.0 - a.b2) * gr * gr;
        m[p] = mm;
        v[p] = vv;
        P[p] -= a.lr * (mm / a.bc1) / (sqrt(vv / a.bc2) + a.eps);
    }
}

// mean over 3na of (F - Fref)^2 added to out[0] (block partials, then one block)
__global__ void __launch_bounds__(256)
k_sg_mse_part(const double* __restrict__ F, const double* __restrict__ Fref, int n3, double* __restrict__ part) {
    __shared__ double sm[32];
    double acc[1] = {0.0};
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n3; e += gridDim.x * blockDim.x) {
        const double d = F[e] - Fref[e];
        acc[0] += d * d;
    }
    block_sum_store<1>(acc, sm, part + blockIdx.x);
}
__global__ void __launch_bounds__(256)
k_sg_mse_final(const double* __restrict__ part, int nblk, int n3, double* __restrict__ out) {
    __shared__ double sm[32];
    double acc[1] = {0.0};
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) acc[0] += part[b];
    double tot[1];
    block_sum_store<1>(acc, sm, tot);
    if (threadIdx.x == 0) out[0] += tot[0] / n3;
}

// Per-feature sums of the (raw) descriptors of rows [0, R): acc[2f] += x,
// acc[2f+1] += x^2.
__global__ void __launch_bounds__(256)
k_sg_xstats(const uint16_t* __restrict__ X, const int* __restrict__ nrows, double* __restrict__ acc) {
    __shared__ double sm[2 * D];
    for (int e = threadIdx.x; e < 2 * D; e += blockDim.x) sm[e] = 0.0;
    __syncthreads();
    const int R = *nrows;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
        const unsigned char* tile = reinterpret_cast<const unsigned char*>(X) + (size_t)(r / TILE) * TILE * D * 2;
        for (int f = 0; f < D; f++) {
            const uint16_t bits = *reinterpret_cast<const uint16_t*>(tile + umma::il_off(r % TILE, f, D));
            const double x = (double)__uint_as_float((uint32_t)bits << 16);
            atomicAdd(&sm[2 * f], x);
            atomicAdd(&sm[2 * f + 1], x * x);
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 2 * D; e += blockDim.x) atomicAdd(&acc[e], sm[e]);
}

__global__ void k_sg_grad_out(const float* __restrict__ g, double scale, double* __restrict__ out) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < NPARAM; p += gridDim.x * blockDim.x)
        out[p] = p < OM ? grad_of(g, p) * scale : 0.0;
}

}  // namespace

cudaError_t train_alloc(TrainWork& tw, const Work& w) {
    if (tw.r_cap >= w.r_cap && tw.na_cap >= w.na_cap) return cudaSuccess;
    train_free(tw);
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    };
    const size_t tb = sizeof(uint16_t) * (size_t)w.r_cap * H;
    uint16_t** bufs[10] = {&tw.t.h1, &tw.t.h2, &tw.t.g1, &tw.t.g2, &tw.t.g3, &tw.t.tb1, &tw.t.tb2,
                           &tw.t.z1, &tw.t.z2, &tw.t.z3};
    for (auto b : bufs) A((void**)b, tb);
    A((void**)&tw.U, sizeof(uint16_t) * (size_t)w.r_cap * D);
    A((void**)&tw.beta, sizeof(float) * (size_t)w.r_cap);
    A((void**)&tw.lamF, sizeof(double) * 3 * (size_t)w.na_cap);
    A((void**)&tw.part, sizeof(double) * kRowBlocks);
    A((void**)&tw.sc, sizeof(double) * 32);
    if (e != cudaSuccess) {
        train_free(tw);
        return e;
    }
    tw.r_cap = w.r_cap;
    tw.na_cap = w.na_cap;
    return cudaSuccess;
}

void train_free(TrainWork& tw) {
    uint16_t* bufs[10] = {tw.t.h1, tw.t.h2, tw.t.g1, tw.t.g2, tw.t.g3, tw.t.tb1, tw.t.tb2, tw.t.z1, tw.t.z2, tw.t.z3};
    for (auto b : bufs) cudaFree(b);
    cudaFree(tw.U); cudaFree(tw.beta); cudaFree(tw.lamF); cudaFree(tw.part); cudaFree(tw.sc);
    tw = TrainWork{};
}

cudaError_t accumulate_grad(Work& w, TrainWork& tw, const uint16_t* img, const float* vec, const double* pos,
                            const double* hh, const int* cnt, const int* list, int cap, int na, const double* Fref,
                            const double* ref10, double wE, double wF, double wW, double* F, double* loss_acc,
                            float* grad, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_sg_chain, cudaFuncAttributeMaxDynamicSharedMemorySize, C_TOTAL);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_sg_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, G_TOTAL);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    cudaError_t e = cudaMemsetAsync(F, 0, sizeof(double) * 3 * (size_t)na, st);
    if (e == cudaSuccess) e = rebo_forces(w, img, vec, pos, hh, cnt, list, cap, na, F, w.part, st);
    if (e == cudaSuccess) e = reduce_partials(w.part, kRowBlocks, kNV, tw.sc, st);           // sc[0..9] = E, W
    if (e != cudaSuccess) return e;
    k_sg_lambda<<<kRowBlocks, 256, 0, st>>>(F, Fref, na, wF, tw.lamF, tw.part);
    e = reduce_partials(tw.part, kRowBlocks, 1, tw.sc + 10, st);                              // sc[10] = sum dF^2
    if (e != cudaSuccess) return e;
    k_sg_loss<<<1, 32, 0, st>>>(tw.sc, ref10, tw.sc + 10, na, wE, wF, wW, tw.sc + 12, loss_acc);   // sc[12..21] = lambdas
    k_sg_adjoint<<<kRowBlocks, 128, 0, st>>>(pos, hh, cnt, list, cap, na, w.aoff, w.row_i, w.row_s, vec, tw.lamF,
                                             tw.sc + 12, w.r_cap, tw.beta, tw.U);
    const int* nrows = w.aoff + w.na_used;
    k_sg_chain<<<kSMs, kThreads, C_TOTAL, st>>>(img, vec, nrows, w.X, tw.U, tw.beta, tw.t,
                                                grad + H * D + 2 * H * H, w.err);
    k_sg_wgrad<<<kSMs, kThreads, G_TOTAL, st>>>(nrows, w.X, tw.U, tw.t, grad, w.err);
    return cudaGetLastError();
}

cudaError_t adam_step(double* P, double* m, double* v, const float* grad, const AdamArgs& a, uint16_t* img,
                      float* vec, cudaStream_t st) {
    k_sg_adam<<<64, 256, 0, st>>>(P, m, v, grad, a);
    return pack_params(P, img, vec, st);
}

cudaError_t force_mse(const double* F, const double* Fref, int na, double* part, double* out, cudaStream_t st) {
    k_sg_mse_part<<<kRowBlocks, 256, 0, st>>>(F, Fref, 3 * na, part);
    k_sg_mse_final<<<1, 256, 0, st>>>(part, kRowBlocks, 3 * na, out);
    return cudaGetLastError();
}

cudaError_t feature_sums(const Work& w, double* acc, cudaStream_t st) {
    k_sg_xstats<<<kSMs * 2, 256, 0, st>>>(w.X, w.aoff + w.na_used, acc);
    return cudaGetLastError();
}

cudaError_t grad_to_params(const float* grad, double scale, double* out, cudaStream_t st) {
    k_sg_grad_out<<<64, 256, 0, st>>>(grad, scale, out);
    return cudaGetLastError();
}

}  // namespace sg
}  // namespace fmd
