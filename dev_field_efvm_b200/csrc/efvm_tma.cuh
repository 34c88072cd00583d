// efvm_tma.cuh — the shared-memory row ring of the TMA-fed stage kernel.
//
// A block of WPB warps owns WPB adjacent strips of 31 columns (124 columns) and
// marches a range of rows.  Each slot of the ring holds one grid row of the
// stage input, 128 columns x 4 planes (the block's columns with two halo
// columns on each side), and the same row of U^n over the block's own 124
// columns (RK stages 2 and 3).  Both arrive by cp.async.bulk.tensor (TMA) from
// tensor maps over this GPU's own state buffers (no multicast) and complete on
// the slot's "full" mbarrier; every warp releases a slot on its "empty"
// mbarrier once it is done with that row, and thread 0 refills it.
//
// Row r of the block's row stream lives in slot (r - first) % RING.  The loop
// of iteration j reads rows j, j+1 and j+2; at its start thread 0 waits until
// every warp has released row j-1 and loads row j-1+RING into that slot, ahead
// of its first use.
//
// Every wait is bounded: one that runs out sets bit 3 of the context's
// nonphysical word (reported as EFVM_ERR_TIMEOUT), and the block stops
// marching; before it exits, thread 0 waits (bounded again) for the copies it
// issued, so that no copy lands in the shared memory of a later block.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace efvm {
namespace tma {

constexpr int RING = 4;                          // row slots (a power of two)
constexpr int IN_COLS = 128;                     // stage-input columns per slot (124 + 2 x 2 halo)
constexpr int U0_COLS = 124;                     // U^n columns per slot (the block's own cells)
constexpr int IN_BYTES = 4 * IN_COLS * 8;        // 4096
constexpr int U0_BYTES = 4 * U0_COLS * 8;        // 3968
// U^n rows in the ring (true), or read from global memory in the epilogue
// (false: 4 KB slots, so more slots or blocks fit the SM's shared memory)
constexpr bool U0_IN_RING = true;
constexpr int SLOT_BYTES = IN_BYTES + (U0_IN_RING ? U0_BYTES : 0);  // 8064 = 63 x 128
constexpr int SMEM_BYTES = RING * SLOT_BYTES + 2 * RING * 8;
constexpr uint32_t WAIT_LIMIT = 1u << 26;        // polls of a wait before it gives up, whatever the time
constexpr int TIMEOUT_BIT = 8;                   // DevState::nonphysical bit of a wait that ran out

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void arrive_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool try_wait(uint64_t* bar, uint32_t parity) {
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
__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait for phase `parity` of *bar: false once limit_ns have passed
// (or WAIT_LIMIT polls, whichever comes first).
__device__ __forceinline__ bool wait(uint64_t* bar, uint32_t parity, unsigned long long limit_ns) {
    if (try_wait(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    for (uint32_t it = 1; it < WAIT_LIMIT; ++it) {
        if (try_wait(bar, parity)) return true;
        if ((it & 31u) == 0u && now_ns() - t0 > limit_ns) return false;
    }
    return false;
}
// One 3-D tile (x, y, plane) of a tensor map into shared memory, completing on *bar.
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void prefetch_map(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

}  // namespace tma
}  // namespace efvm
