// Device helpers shared by the tcgen05 kernels (tc_gemm.cu, mlp.cu):
// mbarriers with waits bounded in time, shared-memory matrix descriptors,
// tcgen05 commit / fences and TMEM loads.
#pragma once

#include <cstdint>

namespace dmrgpp {
namespace tc {

constexpr unsigned long long kWaitNs = 500ull * 1000ull * 1000ull;

__device__ __forceinline__ unsigned smem_addr(const void* p)
{
	return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long now_ns()
{
	unsigned long long t;
	asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
	return t;
}

__device__ __forceinline__ void mbar_init(unsigned addr, unsigned count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(addr), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned addr, unsigned bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(addr), "r"(bytes)
	             : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned addr)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(addr) : "memory");
}

__device__ __forceinline__ bool mbar_try(unsigned addr, unsigned parity)
{
	unsigned ok;
	asm volatile("{\n\t.reg .pred p;\n\t"
	             "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
	             "selp.u32 %0, 1, 0, p;\n\t}\n"
	             : "=r"(ok)
	             : "r"(addr), "r"(parity)
	             : "memory");
	return ok != 0;
}

// true once the phase of the given parity has completed; false after kWaitNs
// or, when abort is given, as soon as *abort is set
__device__ __forceinline__ bool mbar_wait(unsigned addr, unsigned parity, const volatile int* abort)
{
	const unsigned long long t0 = now_ns();
	for (;;) {
		if (mbar_try(addr, parity))
			return true;
		if (abort && *abort)
			return false;
		if (now_ns() - t0 > kWaitNs)
			return false;
	}
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), version 1 (sm_100), base offset 0 (1024-aligned
// tiles); the K step inside a 128-byte row is an address offset
__device__ __forceinline__ uint64_t smem_desc(unsigned saddr)
{
	return (uint64_t((saddr >> 4) & 0x3FFFu)) | (uint64_t(1) << 16) | (uint64_t(1024 >> 4) << 32)
	    | (uint64_t(1) << 46) | (uint64_t(2) << 61);
}

__device__ __forceinline__ void mma_commit(unsigned mbar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
	                 mbar)
	             : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(unsigned taddr, float (&v)[32])
{
	unsigned r[32];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
	             "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
	             "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
	               "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
	               "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
	               "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
	               "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
	               "=r"(r[30]), "=r"(r[31])
	             : "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
	for (int i = 0; i < 32; ++i)
		v[i] = __uint_as_float(r[i]);
}

} // namespace tc
} // namespace dmrgpp
