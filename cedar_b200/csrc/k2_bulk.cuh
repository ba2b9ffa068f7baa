// k2_bulk.cuh -- bulk asynchronous global->shared copies completed on an
// mbarrier (cp.async.bulk, no multicast), with waits bounded by a poll count.
#pragma once
#include <cstdint>

namespace cdrgpu {

static __device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

static __device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

static __device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
	             : "memory");
}

static __device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
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

// at most 2^18 polls (each try_wait may suspend the thread for a while)
static __device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity)
{
	for (int it = 0; it < (1 << 18); ++it)
		if (mbar_try_wait(bar, parity)) return true;
	return false;
}

// global -> shared bulk copy completing on *bar (no multicast); 16-byte aligned
// addresses, size a multiple of 16
static __device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
	                 smem_u32(dst)),
	             "l"(src), "r"(bytes), "r"(smem_u32(bar))
	             : "memory");
}

}  // namespace cdrgpu
