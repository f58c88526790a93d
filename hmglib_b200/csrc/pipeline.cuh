// pipeline.cuh -- shared-memory staging with bulk asynchronous copies (sm_90+/sm_100a).
//
// A producer lane issues cp.async.bulk global->shared copies that complete on an
// mbarrier ("full"); consumer warps wait on it, compute from shared memory and
// arrive on a second mbarrier ("empty") that lets the producer reuse the stage.
// Every wait is bounded by a clock budget: on expiry the waiting thread records
// an error code in a device flag and the kernel unwinds, so a logic error can
// never leave a GPU spinning.
#pragma once

#include <stdint.h>

namespace hmg {

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity; false (and *err set) after ~2^31 cycles.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* err, int code)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > (1ll << 31)) {
            atomicCAS(err, 0, code);
            return false;
        }
    }
    return true;
}

// 1-D bulk copy global -> shared, completing `bytes` of transaction on `bar`.
// dst, src and bytes must be multiples of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// barrier among the consumer warps only (named barrier 1)
__device__ __forceinline__ void consumers_sync(int nthreads)
{
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

}  // namespace hmg
