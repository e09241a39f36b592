// Tensor-memory-accelerator staging for the smoothing kernels: 2D box copies of padded level
// arrays from global into shared memory, completed on a CTA-local mbarrier.
//
// Only plain (non-multicast) loads from this GPU's own memory are issued. Every wait is bounded:
// after kWaitLimit polls a wait reports failure, and its caller records an error and stops.
#pragma once

#include <cstdint>

namespace fc
{

constexpr unsigned kWaitLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_address(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbarrier_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_address(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation and earlier shared-memory accesses of this thread visible to the
// asynchronous (TMA) proxy.
__device__ __forceinline__ void fence_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbarrier_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("{\n\t.reg .b64 state;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 state, [%0], %1;\n\t}" ::"r"(
                     smem_address(bar)),
        "r"(bytes)
        : "memory");
}

// One arrival with no transaction bytes: completes the phase of a barrier of count 1 that is
// given no copies.
__device__ __forceinline__ void mbarrier_arrive(uint64_t* bar)
{
    asm volatile("{\n\t.reg .b64 state;\n\tmbarrier.arrive.shared::cta.b64 state, [%0];\n\t}" ::"r"(smem_address(bar))
                 : "memory");
}

// True once the barrier's phase with the given parity has completed; false after kWaitLimit polls.
__device__ __forceinline__ bool mbarrier_wait(uint64_t* bar, unsigned parity)
{
    const uint32_t addr = smem_address(bar);
    for (unsigned i = 0; i < kWaitLimit; ++i)
    {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(addr), "r"(parity)
                     : "memory");
        if (done)
            return true;
    }
    return false;
}

// One 2D box of a tensor map at element coordinates (x, y) into shared memory; counts its bytes
// on the barrier. Coordinates outside the tensor read as zero.
__device__ __forceinline__ void tma_load_2d(void* dst, const void* map, int x, int y, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_address(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_address(bar))
        : "memory");
}

// A contiguous copy of `bytes` from global into shared memory, counted on the barrier. Both
// addresses must be 16-byte aligned and `bytes` a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_address(dst)),
        "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_address(bar))
        : "memory");
}

__device__ __forceinline__ void prefetch_tensormap(const void* map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

} // namespace fc
