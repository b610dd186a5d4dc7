// umma_selftest.cu -- TEST ONLY (built by fuller_md_en_b200/build.py into
// tests/_build/, never into the product library): one 128 x N x K BF16 GEMM
// through tcgen05.mma with the operands in each major-ness the learned-
// potential kernels use, so tests/test_sg_umma.py pins the descriptor
// conventions of the package's umma.cuh (K-major and MN-major views of the
// interleaved layout) against a CPU product.
#include <cuda_runtime.h>
#include <stdint.h>

#include "umma.cuh"

namespace fmd {
namespace {

using namespace umma;

// A: 128 x K (row-major, bf16 bits), Bt: N x K (row-major), D = A * Bt^T.
// mode bit 0: A read MN-major (stored transposed); bit 1: B read MN-major.
__global__ void __launch_bounds__(128) k_umma_selftest(const uint16_t* __restrict__ A,
                                                       const uint16_t* __restrict__ Bt, int K, int N, int mode,
                                                       float* __restrict__ D, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char* sA = sm;                     // 128 x K  (or K x 128)
    unsigned char* sB = sm + 128 * K * 2;       // N x K    (or K x N)
    __shared__ uint64_t mbar;
    __shared__ uint32_t tbase;
    const int t = threadIdx.x, w = t >> 5;
    const bool amn = mode & 1, bmn = mode & 2;
    for (int e = t; e < 128 * K; e += 128) {
        const int m = e / K, k = e % K;
        const uint32_t off = amn ? il_off(k, m, 128) : il_off(m, k, K);
        *reinterpret_cast<uint16_t*>(sA + off) = A[e];
    }
    for (int e = t; e < N * K; e += 128) {
        const int n = e / K, k = e % K;
        const uint32_t off = bmn ? il_off(k, n, N) : il_off(n, k, K);
        *reinterpret_cast<uint16_t*>(sB + off) = Bt[e];
    }
    if (w == 0) {
        tmem_alloc(&tbase, 256);
        tmem_relinquish();
    }
    if (t == 0) mbar_init(&mbar, 1);
    fence_smem_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tm = tbase;
    if (t == 0) {
        const uint32_t id = idesc_bf16(128, N, amn, bmn);
        const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
        for (int s = 0; s < K / 16; s++) {
            const uint64_t da = amn ? desc_mn(a0, 128, s) : desc_k(a0, K, s);
            const uint64_t db = bmn ? desc_mn(b0, N, s) : desc_k(b0, K, s);
            mma_bf16(tm, da, db, id, s > 0);
        }
        commit(&mbar);
    }
    const bool ok = mbar_wait(&mbar, 0);
    fence_after();
    if (!ok) {
        if (t == 0) atomicExch(err, 1);
    } else {
        const int row = 32 * w + (t & 31);
        for (int c = 0; c < N; c += 16) {
            float v[16];
            tmem_ld16(tm + ((uint32_t)(32 * w) << 16) + c, v);
            for (int q = 0; q < 16; q++) D[(size_t)row * N + c + q] = v[q];
        }
    }
    fence_before();
    __syncthreads();
    if (w == 0) tmem_dealloc(tm, 256);
}

}  // namespace
}  // namespace fmd

// D = A * Bt^T on the current device: A is 128 x K and Bt is N x K,
// row-major bf16 bit patterns; mode bit 0 reads A MN-major and bit 1 reads B
// MN-major from shared memory.  K, N multiples of 16 in [16, 256].
// Returns 0 on success, 1 for bad arguments, 2 for a CUDA error, 3 when the
// kernel's bounded wait for the MMA's completion ran out.
extern "C" int fmd_umma_selftest(const uint16_t* A, const uint16_t* Bt, int K, int N, int mode, float* D) {
    using namespace fmd;
    if (!A || !Bt || !D || K < 16 || K > 256 || K % 16 || N < 16 || N > 256 || N % 16 || mode < 0 || mode > 3)
        return 1;
    uint16_t *dA = nullptr, *dB = nullptr;
    float* dD = nullptr;
    int* dErr = nullptr;
    int herr = 0;
    const size_t smem = (size_t)(128 + N) * K * 2;
    auto cleanup = [&]() {
        cudaFree(dA); cudaFree(dB); cudaFree(dD); cudaFree(dErr);
    };
    if (cudaMalloc(&dA, 128 * (size_t)K * 2) != cudaSuccess || cudaMalloc(&dB, (size_t)N * K * 2) != cudaSuccess ||
        cudaMalloc(&dD, 128 * (size_t)N * 4) != cudaSuccess || cudaMalloc(&dErr, sizeof(int)) != cudaSuccess) {
        cleanup();
        return 2;
    }
    cudaMemcpy(dA, A, 128 * (size_t)K * 2, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, Bt, (size_t)N * K * 2, cudaMemcpyHostToDevice);
    cudaMemset(dErr, 0, sizeof(int));
    cudaFuncSetAttribute(k_umma_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_umma_selftest<<<1, 128, smem>>>(dA, dB, K, N, mode, dD, dErr);
    cudaMemcpy(D, dD, 128 * (size_t)N * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(&herr, dErr, sizeof(int), cudaMemcpyDeviceToHost);
    const cudaError_t e = cudaDeviceSynchronize();
    cleanup();
    if (e != cudaSuccess) return 2;
    return herr ? 3 : 0;
}
