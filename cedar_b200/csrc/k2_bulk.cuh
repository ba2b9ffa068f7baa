// k2_bulk.cuh -- bulk asynchronous global->shared copies completed on an
// mbarrier (cp.async.bulk, no multicast), with waits bounded in time.
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

static __device__ __forceinline__ unsigned long long globaltimer_ns()
{
	unsigned long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// Default limits of the bounded waits: the first wait of a streamed kernel on
// a stage, and the drain of a CTA that gave up (its copies still in flight).
constexpr unsigned long long kWaitLimitNs = 200000000ull;   // 0.2 s
constexpr unsigned long long kDrainLimitNs = 1000000000ull; // 1 s

// Wait for the phase of `parity` to complete, for at most limit_ns
// nanoseconds of the global timer (and at most 2^20 polls); limit_ns = 0 gives
// up at once (the test setting of the give-up path).  Returns false if it gave up.
static __device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity,
                                                         unsigned long long limit_ns = kWaitLimitNs)
{
	if (limit_ns == 0) return false;
	const unsigned long long t0 = globaltimer_ns();
	for (int it = 0; it < (1 << 20); ++it) {
		if (mbar_try_wait(bar, parity)) return true;
		if (globaltimer_ns() - t0 > limit_ns) return false;
	}
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
