// Mixed-precision grouped GEMM on the 5th-generation tensor cores (tcgen05).
//
// TF32x3: each FP64 operand is carried as two TF32 parts, a = a_hi + a_lo, and
// one tile accumulates a_hi*b_hi + a_hi*b_lo + a_lo*b_hi in FP32 in tensor
// memory (the a_lo*b_lo term is below the FP32 accumulation error).
//
// One CTA (4 warps) computes a 128 x BN output tile of a grouped pass
// (kron_plan.h, MixedPlan): for every K-segment of the tile, 32-wide k-chunks
// of A (128 rows) and B (BN rows), both K-major and split into hi/lo, are
// staged by cp.async into shared memory in the 128-byte-swizzled K-major
// layout that tcgen05.mma reads through shared-memory descriptors; thread 0
// issues 3 x 4 MMAs (M=128, N=BN, K=8) per chunk into one TMEM accumulator
// and commits them to the chunk's mbarrier, which frees the stage for the
// next load.  The epilogue reads the accumulator with tcgen05.ld (warp w owns
// TMEM lanes 32w..32w+31 = tile rows) and either splits it again into hi/lo
// (pass 1, the A operand of pass 2) or widens it to FP64 (pass 2, y).
//
// Every mbarrier wait is bounded in time; a wait that gives up sets the
// error word, waits (bounded) for the tensor core once more, frees TMEM and
// leaves the tile unwritten.
#include "tc_gemm.cuh"

#include <cstdint>

namespace dmrgpp {
namespace {

constexpr int                kBM         = 128;
constexpr int                kBK         = 32; // TF32 elements = 128 bytes per row per chunk
constexpr unsigned long long kWaitNs     = 500ull * 1000ull * 1000ull;
constexpr int                kTcThreads  = 128;

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

__device__ __forceinline__ void cp_async_16(unsigned dst, const void* src, bool pred)
{
	const int n = pred ? 16 : 0;
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n)
	             : "memory");
}

__device__ __forceinline__ void cp_async_commit()
{
	asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int N> __device__ __forceinline__ void cp_async_wait()
{
	asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void mbar_init(unsigned addr, unsigned count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(addr), "r"(count) : "memory");
}

// true once the phase of the given parity has completed; false after kWaitNs
__device__ __forceinline__ bool mbar_wait(unsigned addr, unsigned parity)
{
	const unsigned long long t0 = now_ns();
	for (;;) {
		unsigned ok;
		asm volatile("{\n\t.reg .pred p;\n\t"
		             "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		             "selp.u32 %0, 1, 0, p;\n\t}\n"
		             : "=r"(ok)
		             : "r"(addr), "r"(parity)
		             : "memory");
		if (ok)
			return true;
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

// instruction descriptor, kind::tf32: D = F32, A = B = TF32, both K-major
template <int BN> __device__ __forceinline__ unsigned idesc_tf32()
{
	return (1u << 4) | (2u << 7) | (2u << 10) | (unsigned(BN >> 3) << 17) | (unsigned(kBM >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(unsigned d, uint64_t a, uint64_t b, unsigned idesc, unsigned acc)
{
	asm volatile("{\n\t.reg .pred p;\n\t"
	             "setp.ne.b32 p, %4, 0;\n\t"
	             "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
	             "l"(a), "l"(b), "r"(idesc), "r"(acc)
	             : "memory");
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

__device__ __forceinline__ float tf32_rna(float f)
{
	unsigned u;
	asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(u) : "f"(f));
	return __uint_as_float(u);
}

template <int BN> struct TcLayout {
	static constexpr int A_BYTES     = kBM * 128;
	static constexpr int B_BYTES     = BN * 128;
	static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
};

// one 32-wide k-chunk of the hi/lo A (128 rows) and B (BN rows) tiles,
// 16-byte pieces placed at chunk ^ (row % 8) inside each 128-byte row
template <int BN>
__device__ __forceinline__ void load_chunk(unsigned stage, const TcArgs& a, const GemmSeg& sg, int k0,
                                           const GemmTile& t)
{
	using L = TcLayout<BN>;
	constexpr int A_PIECES = kBM * 8 / kTcThreads;
	constexpr int B_PIECES = BN * 8 / kTcThreads;
#pragma unroll
	for (int e = 0; e < A_PIECES; ++e) {
		const int      idx  = threadIdx.x + e * kTcThreads;
		const int      row  = idx >> 3;
		const int      c    = idx & 7;
		const bool     p    = t.m0 + row < t.M;
		const long long off = sg.a_off + (long long)(t.m0 + (p ? row : 0)) * sg.lda + k0 + c * 4;
		const unsigned dst  = unsigned(row * 128 + ((c ^ (row & 7)) << 4));
		cp_async_16(stage + dst, a.A_hi + off, p);
		cp_async_16(stage + L::A_BYTES + dst, a.A_lo + off, p);
	}
#pragma unroll
	for (int e = 0; e < B_PIECES; ++e) {
		const int      idx  = threadIdx.x + e * kTcThreads;
		const int      row  = idx >> 3;
		const int      c    = idx & 7;
		const bool     p    = t.n0 + row < t.N;
		const long long off = sg.b_off + (long long)(t.n0 + (p ? row : 0)) * sg.ldb + k0 + c * 4;
		const unsigned dst  = unsigned(row * 128 + ((c ^ (row & 7)) << 4));
		cp_async_16(stage + 2 * L::A_BYTES + dst, a.B_hi + off, p);
		cp_async_16(stage + 2 * L::A_BYTES + L::B_BYTES + dst, a.B_lo + off, p);
	}
}

template <int BN, int STAGES, bool PASS1>
__global__ void __launch_bounds__(kTcThreads) tc_gemm_tf32x3_kernel(TcArgs a)
{
	using L = TcLayout<BN>;
	extern __shared__ unsigned char smem_raw[];
	__shared__ __align__(8) unsigned long long mbar[STAGES];
	__shared__ unsigned                        tmem_slot;

	const unsigned base = (smem_addr(smem_raw) + 1023u) & ~1023u; // 1024-aligned stages
	const GemmTile t    = a.tiles[blockIdx.x];
	const int      tid  = threadIdx.x;
	const int      warp = tid >> 5;
	const int      lane = tid & 31;

	if (warp == 0) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
		                 smem_addr(&tmem_slot)),
		             "r"(unsigned(BN))
		             : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
	}
	if (tid == 0) {
		for (int s = 0; s < STAGES; ++s)
			mbar_init(smem_addr(&mbar[s]), 1);
		asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const unsigned tmem = tmem_slot;

	int total = 0;
	for (int s = t.seg_begin; s < t.seg_end; ++s)
		total += (a.segs[s].K + kBK - 1) / kBK;

	int     ls = t.seg_begin, lk = 0;
	GemmSeg cur {};
	if (ls < t.seg_end)
		cur = a.segs[ls];
	auto issue = [&](int stage) {
		load_chunk<BN>(base + unsigned(stage * L::STAGE_BYTES), a, cur, lk, t);
		lk += kBK;
		if (lk >= cur.K) {
			lk = 0;
			if (++ls < t.seg_end)
				cur = a.segs[ls];
		}
	};

#pragma unroll
	for (int st = 0; st < STAGES - 1; ++st) {
		if (st < total)
			issue(st);
		cp_async_commit();
	}
	bool           ok     = true;
	int            issued = 0; // chunks whose MMAs were committed
	const unsigned idesc  = idesc_tf32<BN>();
	for (int it = 0; it < total; ++it) {
		cp_async_wait<STAGES - 2>();
		asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
		ok = __syncthreads_and(ok) != 0; // uniform: a timed-out wait stops every thread
		if (!ok)
			break;
		if (tid == 0) {
			tc_fence_after();
			const unsigned sa = base + unsigned((it % STAGES) * L::STAGE_BYTES);
			const unsigned ahi = sa, alo = sa + L::A_BYTES;
			const unsigned bhi = sa + 2 * L::A_BYTES, blo = bhi + L::B_BYTES;
#pragma unroll
			for (int ks = 0; ks < kBK / 8; ++ks) {
				const unsigned kb = unsigned(ks * 32); // 8 TF32 = 32 bytes along K
				mma_tf32(tmem, smem_desc(ahi + kb), smem_desc(bhi + kb), idesc, (it | ks) != 0);
				mma_tf32(tmem, smem_desc(ahi + kb), smem_desc(blo + kb), idesc, 1u);
				mma_tf32(tmem, smem_desc(alo + kb), smem_desc(bhi + kb), idesc, 1u);
			}
			mma_commit(smem_addr(&mbar[it % STAGES]));
		}
		issued = it + 1;
		const int nxt = it + STAGES - 1;
		if (nxt < total) {
			// the target stage was last read by the MMAs of chunk it-1
			if (it >= 1)
				ok = mbar_wait(smem_addr(&mbar[(it - 1) % STAGES]), unsigned(((it - 1) / STAGES) & 1))
				    && ok;
			issue(nxt % STAGES);
		}
		cp_async_commit();
	}
	cp_async_wait<0>();
	// the last commit covers every MMA issued before it; after a timeout this
	// is the (bounded) drain before TMEM is read or freed
	if (issued > 0 && !mbar_wait(smem_addr(&mbar[(issued - 1) % STAGES]),
	                             unsigned(((issued - 1) / STAGES) & 1)))
		ok = false;
	ok = __syncthreads_and(ok) != 0;
	tc_fence_after();
	if (!ok)
		atomicExch(a.error, 2);

	// epilogue: warp w holds tile rows 32w..32w+31 (TMEM lanes)
	const int row  = warp * 32 + lane;
	const int grow = t.m0 + row;
	for (int c0 = 0; c0 < BN; c0 += 32) {
		float v[32];
		if (total > 0) {
			tmem_ld32(tmem + (unsigned(warp * 32) << 16) + unsigned(c0), v);
		} else {
#pragma unroll
			for (int i = 0; i < 32; ++i)
				v[i] = 0.f;
		}
		if (!ok || grow >= t.M || t.n0 + c0 >= t.N)
			continue;
		if (PASS1) {
			// K-major row of the next pass; columns past N carry exact zeros
			// (zero-filled B rows), which keep the K padding zero
			float*          hi  = a.C_hi + t.c_off + (long long)grow * t.ldc + t.n0 + c0;
			float*          lo  = a.C_lo + t.c_off + (long long)grow * t.ldc + t.n0 + c0;
#pragma unroll
			for (int q = 0; q < 8; ++q) {
				float4 h, l;
				h.x = tf32_rna(v[4 * q + 0]);
				h.y = tf32_rna(v[4 * q + 1]);
				h.z = tf32_rna(v[4 * q + 2]);
				h.w = tf32_rna(v[4 * q + 3]);
				l.x = tf32_rna(v[4 * q + 0] - h.x);
				l.y = tf32_rna(v[4 * q + 1] - h.y);
				l.z = tf32_rna(v[4 * q + 2] - h.z);
				l.w = tf32_rna(v[4 * q + 3] - h.w);
				reinterpret_cast<float4*>(hi)[q] = h;
				reinterpret_cast<float4*>(lo)[q] = l;
			}
		} else {
			double* y = a.Cd + t.c_off;
#pragma unroll
			for (int i = 0; i < 32; ++i) {
				const int gcol = t.n0 + c0 + i;
				if (gcol < t.N)
					y[(long long)gcol * t.ldc + grow] = double(v[i]);
			}
		}
	}

	tc_fence_before();
	__syncthreads();
	if (warp == 0)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
		             "r"(unsigned(BN))
		             : "memory");
}

// x (FP64, patch order) -> K-major TF32 hi/lo split buffers
__global__ void __launch_bounds__(256)
split_x_kernel(const double* __restrict__ x, const int* __restrict__ map, float* __restrict__ hi,
               float* __restrict__ lo, long long n)
{
	for (long long e = blockIdx.x * 256LL + threadIdx.x; e < n; e += 256LL * gridDim.x) {
		const double v = x[e];
		const float  h = tf32_rna(float(v));
		const int    d = map[e];
		hi[d]          = h;
		lo[d]          = tf32_rna(float(v - double(h)));
	}
}

template <int BN, int STAGES, bool PASS1> constexpr size_t tc_smem()
{
	return size_t(STAGES) * TcLayout<BN>::STAGE_BYTES + 1024;
}

template <int BN, int STAGES, bool PASS1> cudaError_t tc_init_one()
{
	return cudaFuncSetAttribute(tc_gemm_tf32x3_kernel<BN, STAGES, PASS1>,
	                            cudaFuncAttributeMaxDynamicSharedMemorySize,
	                            int(tc_smem<BN, STAGES, PASS1>()));
}

} // namespace

cudaError_t tc_init()
{
	cudaError_t e = tc_init_one<64, 3, true>();
	if (e == cudaSuccess)
		e = tc_init_one<64, 3, false>();
	if (e == cudaSuccess)
		e = tc_init_one<128, 3, true>();
	if (e == cudaSuccess)
		e = tc_init_one<128, 3, false>();
	return e;
}

cudaError_t tc_launch(const TcArgs& a, int bn, bool pass1, cudaStream_t stream)
{
	if (a.ntiles <= 0)
		return cudaSuccess;
	if (bn == 64) {
		if (pass1)
			tc_gemm_tf32x3_kernel<64, 3, true><<<a.ntiles, kTcThreads, tc_smem<64, 3, true>(), stream>>>(a);
		else
			tc_gemm_tf32x3_kernel<64, 3, false><<<a.ntiles, kTcThreads, tc_smem<64, 3, false>(), stream>>>(a);
	} else if (bn == 128) {
		if (pass1)
			tc_gemm_tf32x3_kernel<128, 3, true><<<a.ntiles, kTcThreads, tc_smem<128, 3, true>(), stream>>>(a);
		else
			tc_gemm_tf32x3_kernel<128, 3, false><<<a.ntiles, kTcThreads, tc_smem<128, 3, false>(), stream>>>(a);
	} else {
		return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

cudaError_t tc_split_x(const double* x, const int* map, float* hi, float* lo, long long n,
                       cudaStream_t stream)
{
	if (n <= 0)
		return cudaSuccess;
	long long blocks = (n + 255) / 256;
	if (blocks > 148 * 8)
		blocks = 148 * 8;
	split_x_kernel<<<int(blocks), 256, 0, stream>>>(x, map, hi, lo, n);
	return cudaGetLastError();
}

} // namespace dmrgpp
