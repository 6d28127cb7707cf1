// async.cuh -- cp.async (global -> shared, 16 bytes, bypassing L1) helpers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace p2g {

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
// waits until at most N of this thread's committed groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

}  // namespace p2g
