// Device building blocks shared by the FP64 grouped-GEMM kernels: one
// CTA-tile of C(BM x BN) = sum over K-segments of A(M x K) * B(K x N) on the
// FP64 tensor pipe (mma.sync m8n8k4 .f64), with operands staged global ->
// shared by cp.async in a STAGES-deep ring.
#pragma once

#include "kron_plan.h"

#include <cuda_runtime.h>

namespace dmrgpp {
namespace tile {

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
	return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// 8-byte asynchronous global->shared copy; src_bytes = 0 zero-fills the
// destination without reading the source.
__device__ __forceinline__ void cp_async_8(unsigned dst, const double* src, bool pred)
{
	const int n = pred ? 8 : 0;
	asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(n)
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

// D(8x8) += A(8x4) * B(4x8) on the FP64 tensor pipe.  Fragments: lane holds
// A[lane/4][lane%4], B[lane%4][lane/4], and C/D[lane/4][2*(lane%4) + {0,1}].
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b)
{
	asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
	             : "+d"(d0), "+d"(d1)
	             : "d"(a), "d"(b));
}

template <int BM_, int BN_, int BK_, int WM_, int WN_, int STAGES_> struct Cfg {
	static constexpr int BM = BM_, BN = BN_, BK = BK_, WM = WM_, WN = WN_, STAGES = STAGES_;
	static constexpr int WARPS_M = BM / WM, WARPS_N = BN / WN;
	static constexpr int THREADS = WARPS_M * WARPS_N * 32;
	static constexpr int MI = WM / 8, NI = WN / 8;
	// shared layouts As[k][m] and Bs[n][k]; the +4 padding makes a warp's
	// fragment reads hit every bank pair exactly twice (the minimum for 256 B)
	static constexpr int LDA_S = BM + 4;
	static constexpr int LDB_S = BK + 4;
	static constexpr int A_STAGE = BK * LDA_S;
	static constexpr int B_STAGE = BN * LDB_S;
	static constexpr size_t SMEM = size_t(STAGES) * (A_STAGE + B_STAGE) * sizeof(double);
	static constexpr int A_LOADS = BM * BK / THREADS;
	static constexpr int B_LOADS = BK * BN / THREADS;
	static_assert(BM * BK % THREADS == 0 && BK * BN % THREADS == 0, "load split");
	static_assert(BK % 4 == 0 && WM % 8 == 0 && WN % 8 == 0, "mma shape");
};

template <class C> struct Acc {
	double v[C::MI][C::NI][2];
};

template <class C>
__device__ __forceinline__ void load_stage(double*       As,
                                           double*       Bs,
                                           const double* A,
                                           int           lda,
                                           const double* B,
                                           int           ldb,
                                           int           K,
                                           int           k0,
                                           int           m0,
                                           int           n0,
                                           int           M,
                                           int           N,
                                           int           tid)
{
#pragma unroll
	for (int e = 0; e < C::A_LOADS; ++e) {
		const int     idx = tid + e * C::THREADS;
		const int     m   = idx % C::BM;
		const int     kk  = idx / C::BM;
		const int     gm  = m0 + m;
		const int     gk  = k0 + kk;
		const bool    p   = gm < M && gk < K;
		const double* src = p ? A + (long long)gk * lda + gm : A;
		cp_async_8(smem_u32(As + kk * C::LDA_S + m), src, p);
	}
#pragma unroll
	for (int e = 0; e < C::B_LOADS; ++e) {
		const int     idx = tid + e * C::THREADS;
		const int     kk  = idx % C::BK;
		const int     n   = idx / C::BK;
		const int     gk  = k0 + kk;
		const int     gn  = n0 + n;
		const bool    p   = gk < K && gn < N;
		const double* src = p ? B + (long long)gn * ldb + gk : B;
		cp_async_8(smem_u32(Bs + n * C::LDB_S + kk), src, p);
	}
}

// acc = sum over segments [sb, se) of A_s[m0.., :] * B_s[:, n0..].
// smem must hold C::SMEM bytes; on return every cp.async of this CTA has
// completed and all threads have passed a barrier after the last shared read.
template <class C>
__device__ __forceinline__ void mma_tile(Acc<C>&        acc,
                                         double*        smem,
                                         const double*  Abase,
                                         const double*  Bbase,
                                         const GemmSeg* segs,
                                         int            sb,
                                         int            se,
                                         int            m0,
                                         int            n0,
                                         int            M,
                                         int            N)
{
	double*   As   = smem;
	double*   Bs   = smem + C::STAGES * C::A_STAGE;
	const int tid  = threadIdx.x;
	const int lane = tid & 31;
	const int warp = tid >> 5;
	const int wm   = warp % C::WARPS_M;
	const int wn   = warp / C::WARPS_M;

#pragma unroll
	for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
		for (int ni = 0; ni < C::NI; ++ni)
			acc.v[mi][ni][0] = acc.v[mi][ni][1] = 0.0;

	int total = 0;
	for (int s = sb; s < se; ++s)
		total += (segs[s].K + C::BK - 1) / C::BK;

	int     ls = sb;
	int     lk = 0;
	GemmSeg cur {};
	if (ls < se)
		cur = segs[ls];
	auto issue = [&](int stage) {
		load_stage<C>(As + stage * C::A_STAGE,
		              Bs + stage * C::B_STAGE,
		              Abase + cur.a_off,
		              cur.lda,
		              Bbase + cur.b_off,
		              cur.ldb,
		              cur.K,
		              lk,
		              m0,
		              n0,
		              M,
		              N,
		              tid);
		lk += C::BK;
		if (lk >= cur.K) {
			lk = 0;
			++ls;
			if (ls < se)
				cur = segs[ls];
		}
	};

#pragma unroll
	for (int st = 0; st < C::STAGES - 1; ++st) {
		if (st < total)
			issue(st);
		cp_async_commit();
	}

	for (int it = 0; it < total; ++it) {
		cp_async_wait<C::STAGES - 2>();
		__syncthreads();
		const int nxt = it + C::STAGES - 1;
		if (nxt < total)
			issue(nxt % C::STAGES);
		cp_async_commit();

		const double* as = As + (it % C::STAGES) * C::A_STAGE + wm * C::WM + (lane >> 2);
		const double* bs = Bs + (it % C::STAGES) * C::B_STAGE + (wn * C::WN + (lane >> 2)) * C::LDB_S;
#pragma unroll
		for (int ks = 0; ks < C::BK; ks += 4) {
			double af[C::MI], bf[C::NI];
#pragma unroll
			for (int mi = 0; mi < C::MI; ++mi)
				af[mi] = as[(ks + (lane & 3)) * C::LDA_S + mi * 8];
#pragma unroll
			for (int ni = 0; ni < C::NI; ++ni)
				bf[ni] = bs[ni * 8 * C::LDB_S + ks + (lane & 3)];
#pragma unroll
			for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
				for (int ni = 0; ni < C::NI; ++ni)
					dmma_8x8x4(acc.v[mi][ni][0], acc.v[mi][ni][1], af[mi], bf[ni]);
		}
	}
	cp_async_wait<0>();
	__syncthreads(); // shared ring free for the next tile of this CTA
}

// Row and column, inside the tile, of accumulator element (mi, ni, h).
template <class C> __device__ __forceinline__ int acc_row(int mi)
{
	const int warp = threadIdx.x >> 5;
	return (warp % C::WARPS_M) * C::WM + mi * 8 + ((threadIdx.x & 31) >> 2);
}
template <class C> __device__ __forceinline__ int acc_col(int ni, int h)
{
	const int warp = threadIdx.x >> 5;
	return (warp / C::WARPS_M) * C::WN + ni * 8 + (threadIdx.x & 3) * 2 + h;
}

} // namespace tile
} // namespace dmrgpp
