// Shared-memory staging by bulk copies (the Blackwell/Hopper TMA unit's
// untiled form, cp.async.bulk) completed on an mbarrier, sm_100a.
//
// A stage is armed by one producer thread with the total byte count of the
// copies it is about to issue (mbarrier.arrive.expect_tx: the barrier's single
// arrival), then each copy signals its bytes on the barrier
// (mbarrier::complete_tx); consumers wait on the stage's phase parity.  Every
// copy moves whole 16-byte units between 16-byte-aligned addresses.  Each CTA
// copies from this GPU's own memory into its own shared memory only.
//
// Waits are bounded: a wait that has not seen its phase complete after about
// two seconds of clock cycles gives up and reports it, so a protocol fault
// surfaces as a status bit instead of a hung GPU.
#pragma once

#include <cstdint>

namespace nimbus
{

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned arrivals)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(arrivals) : "memory");
}

// Makes barrier initialisation visible to the async proxy (the copy engine).
__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_invalidate(uint64_t* bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// The producer's arrival, announcing `bytes` of copies for this phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// dst (shared) <- src (global), `bytes` a multiple of 16, both 16-byte
// aligned; completes `bytes` of transactions on bar.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

constexpr long long kStageWaitCycles = 4000000000LL;  // about two seconds at the boost clock

// Waits for the phase of `parity` to complete; false if it did not within
// kStageWaitCycles.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long start = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - start > kStageWaitCycles) return false;
    return true;
}

// A run of consecutive cells [a, b) of one field, clipped to [0, n) and
// widened to 16-byte units: [lo, hi), hi <= lo when empty.  Member fields are
// padded to 256 bytes, so hi (at most n + 3) stays inside the allocation.
struct CellRun
{
    int lo, hi;
};

__device__ __forceinline__ CellRun cell_run(long long a, long long b, int n)
{
    const long long s = a < 0 ? 0 : a;
    const long long e = b < n ? b : n;
    if (e <= s) return CellRun{0, 0};
    return CellRun{static_cast<int>(s) & ~3, (static_cast<int>(e) + 3) & ~3};
}

}  // namespace nimbus
