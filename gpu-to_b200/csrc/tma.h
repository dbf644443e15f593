// Tensor Memory Accelerator (TMA) helpers for sm_100a: tensor-map encoding on
// the host and the PTX for tile loads completed on an mbarrier.  Only plain
// (non-multicast) tile loads of this GPU's own memory are used.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace gputo {

// Encode a 3-D tiled tensor map over a row-padded array of doubles, floats or
// bytes (elem_bytes 8, 4 or 1):
//   dims (inner, mid, outer) in elements, byte strides of mid and outer,
//   box (b0, b1, b2) in elements.  Out-of-range elements of a box read as 0.
// Returns 0 on success.
int make_tmap_3d(CUtensorMap *m, const void *base, int elem_bytes, uint64_t d0, uint64_t d1,
                 uint64_t d2, uint64_t stride1_bytes, uint64_t stride2_bytes, uint32_t b0,
                 uint32_t b1, uint32_t b2);

#if defined(__CUDACC__)
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

// Make the initialised barrier visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *tm, int c0, int c1, int c2,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase: gives up after 'limit' polls (each poll
// may itself suspend for a bounded, hardware-defined time).  Returns true when
// the phase completed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t limit)
{
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait on an mbarrier phase by elapsed time: gives up after about
// 'limit_ns' nanoseconds of the device's global timer (and after 2^26 polls
// in any case).  Returns true when the phase completed.
__device__ __forceinline__ bool mbar_wait_for(uint64_t *bar, uint32_t parity, uint32_t limit_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > (uint64_t)limit_ns) return false;
    }
    return false;
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *tm)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tm)) : "memory");
}
#endif

}  // namespace gputo
