// umma.cuh -- thin sm_100a wrappers for the 5th-generation tensor cores
// (tcgen05.mma kind::f16, BF16 operands, FP32 accumulators in TMEM),
// the TMEM allocator, TMEM loads and mbarrier waits with iteration limits.
//
// Shared-memory operand layout used everywhere ("interleaved", no swizzle):
// a matrix of R rows x C columns (C contiguous in the math sense) is stored
// as 8x8 core matrices of 16-bit elements,
//     byte(r, c) = (r/8)*S + (c/8)*128 + (r%8)*16 + (c%8)*2,   S = (C/8)*128.
// Read as a K-major operand (rows = M or N, columns = K) its descriptor has
// LBO = 128 (next 8 columns) and SBO = S (next 8 rows).  The SAME bytes read
// as an MN-major operand describe the transpose (rows = K, columns = M/N)
// with SBO = 128 and LBO = S.  So one copy of each weight matrix serves the
// forward GEMM (W) and the backward GEMM (W^T), and an activation tile
// stored for the next layer also serves as the transposed operand of a
// weight-gradient GEMM.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

namespace fmd {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, c) in the interleaved layout with C columns.
__host__ __device__ __forceinline__ uint32_t il_off(int r, int c, int C) {
    return (uint32_t)((r >> 3) * (C >> 3) * 128 + (c >> 3) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

// Shared-memory matrix descriptor (version 1, SWIZZLE_NONE, base offset 0).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// K-major operand: tile with C columns, K-step s (16 columns) starts 256*s bytes in.
__device__ __forceinline__ uint64_t desc_k(uint32_t base, int C, int s) {
    return sdesc(base + 256u * s, 128u, (uint32_t)(C >> 3) * 128u);
}
// MN-major view of a tile stored with C columns and R rows: the MMA's K runs
// over the tile's rows; K-step s starts at row 16*s.
__device__ __forceinline__ uint64_t desc_mn(uint32_t base, int C, int s) {
    const uint32_t S = (uint32_t)(C >> 3) * 128u;
    return sdesc(base + 2u * S * s, S, 128u);
}

// Instruction descriptor, kind::f16: BF16 x BF16 -> FP32, dense.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
// Arrive on *mbar when every tcgen05.mma issued so far by this thread is done.
__device__ __forceinline__ void commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {   // whole warp
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {   // whole warp
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy smem writes -> visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 lanes x 16 consecutive 32-bit columns: thread t of the warp gets lane
// (lane base + t).  The lane base must be 32 * (warp id % 4).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}

// The store of the same shape: thread t of the warp writes lane (lane base +
// t), 16 consecutive columns.  tmem_wait_st() waits for this thread's stores.
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float* v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
        "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
        "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])),
        "r"(__float_as_uint(v[11])), "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])),
        "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* m, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(m)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: false after ~0.5 s (or 2^24 polls), so a lost arrival ends
// the kernel with an error status instead of a hang.
__device__ __forceinline__ bool mbar_wait(uint64_t* m, uint32_t parity) {
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 0; it < (1u << 24); it++) {
        if (mbar_try_wait(m, parity)) return true;
        if ((it & 255u) == 255u && globaltimer_ns() - t0 > 500000000ull) break;
    }
    return false;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const uint32_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(a));
    const uint32_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(b));
    return lo | (hi << 16);
}

}  // namespace umma
}  // namespace fmd
