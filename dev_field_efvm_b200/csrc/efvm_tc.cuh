// efvm_tc.cuh — the 5th-generation tensor-core (tcgen05) building blocks of the
// learned flux correction: tensor-memory allocation, shared-memory matrix
// descriptors, the BF16 x BF16 -> FP32 MMA issued by one thread, its
// completion through an mbarrier, and the accumulator read-back.
//
// Operands live in shared memory in the canonical K-major layout without
// swizzle: an R x K BF16 matrix (R a multiple of 8, K of 16) is a grid of
// "core matrices" of 8 rows x 16 bytes (8 elements of K), each stored as 128
// contiguous bytes; core matrices adjacent in R are SBO = 128 bytes apart and
// those adjacent in K are LBO = 16 * R bytes apart:
//     byte(r, k) = (k / 8) * 16 R + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.
// One MMA consumes K = 16 (two core matrices along K); step s starts at
// 2 s LBO.  The accumulator D (M = 128 rows) occupies TMEM lane r, column j
// for element (r, j), 32 bits each.
//
// Every wait is bounded: a wait that runs out records an error code and the
// kernel carries on to its clean-up (TMEM is always released).
#pragma once

#include <cstdint>

namespace efvm {
namespace tc {

constexpr uint32_t WAIT_LIMIT = 1u << 24;  // mbarrier polls before giving up (far above any real wait)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, k) of an R-row canonical K-major operand.
__device__ __host__ __forceinline__ uint32_t canon_offset(int r, int k, int rows) {
    return (uint32_t)((k >> 3) * 16 * rows + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (sm_100): start address, leading and stride
// byte offsets (all >> 4), version 1 at bits 46-47, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, both K-major,
// M = 128, N (multiple of 16, 16..256).
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int m, int n) {
    return (1u << 4)                       // D format F32
           | (1u << 7)                     // A format BF16
           | (1u << 10)                    // B format BF16
           | ((uint32_t)(n >> 3) << 17)    // N >> 3
           | ((uint32_t)(m >> 4) << 24);   // M >> 4
}

// ---- tensor memory -------------------------------------------------------
// Allocation and release by one whole warp; the TMEM address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Make generic-proxy writes of shared memory visible to the tensor core.
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- mbarrier --------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Bounded wait for the phase `parity` of *bar; false if it ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t it = 0; it < WAIT_LIMIT; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// ---- MMA ---------------------------------------------------------------------
// D (+)= A * B^T for one K = 16 step; one thread issues it.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"((uint32_t)accumulate));
}
// Arrive on *bar once every MMA this thread issued before has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// D[128 x N] = A[128 x K] * B[N x K]^T with A, B canonical in shared memory
// (A has 128 rows, B has N rows), issued by thread 0 and committed to *bar.
__device__ __forceinline__ void gemm_issue(uint32_t tmem_d, const void* a, const void* b, int n, int k,
                                           uint64_t* bar) {
    if (threadIdx.x == 0) {
        fence_after_sync();
        const uint32_t idesc = idesc_bf16_f32(128, n);
        const uint32_t sa = smem_u32(a), sb = smem_u32(b);
        const uint32_t lbo_a = 16u * 128u, lbo_b = 16u * (uint32_t)n;
        for (int s = 0; s < k / 16; ++s) {
            const uint64_t da = smem_desc(sa + 2u * (uint32_t)s * lbo_a, lbo_a, 128u);
            const uint64_t db = smem_desc(sb + 2u * (uint32_t)s * lbo_b, lbo_b, 128u);
            mma_bf16(tmem_d, da, db, idesc, s > 0);
        }
        mma_commit(bar);
    }
}

// ---- accumulator read-back -------------------------------------------------
// Thread t of warp w (w < 4) receives row 32 w + t, columns col0 .. col0 + 15.
__device__ __forceinline__ void tmem_ld16(uint32_t tmem, int col0, float (&v)[16]) {
    const int w = (threadIdx.x >> 5) & 3;
    const uint32_t addr = tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)col0;
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace efvm
