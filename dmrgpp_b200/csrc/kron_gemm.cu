// FP64 grouped GEMM for the two Kronecker passes (see kron_gemm.cuh).
#include "kron_gemm.cuh"

namespace dmrgpp {
namespace {

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

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

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

template <int BM_, int BN_, int BK_, int WM_, int WN_, int STAGES_> struct TileCfg {
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

template <class C>
__device__ __forceinline__ void load_stage(double*        As,
                                           double*        Bs,
                                           const double*  A,
                                           int            lda,
                                           const double*  B,
                                           int            ldb,
                                           int            K,
                                           int            k0,
                                           const GemmTile& t,
                                           int            tid)
{
#pragma unroll
	for (int e = 0; e < C::A_LOADS; ++e) {
		const int  idx = tid + e * C::THREADS;
		const int  m   = idx % C::BM;
		const int  kk  = idx / C::BM;
		const int  gm  = t.m0 + m;
		const int  gk  = k0 + kk;
		const bool p   = gm < t.M && gk < K;
		const double* src = p ? A + (long long)gk * lda + gm : A;
		cp_async_8(smem_u32(As + kk * C::LDA_S + m), src, p);
	}
#pragma unroll
	for (int e = 0; e < C::B_LOADS; ++e) {
		const int  idx = tid + e * C::THREADS;
		const int  kk  = idx % C::BK;
		const int  n   = idx / C::BK;
		const int  gk  = k0 + kk;
		const int  gn  = t.n0 + n;
		const bool p   = gk < K && gn < t.N;
		const double* src = p ? B + (long long)gn * ldb + gk : B;
		cp_async_8(smem_u32(Bs + n * C::LDB_S + kk), src, p);
	}
}

template <class C>
__global__ void __launch_bounds__(C::THREADS) grouped_dgemm_kernel(GemmArgs args)
{
	extern __shared__ __align__(16) double smem[];
	double* As = smem;
	double* Bs = smem + C::STAGES * C::A_STAGE;

	const GemmTile t    = args.tiles[blockIdx.x];
	const int      tid  = threadIdx.x;
	const int      lane = tid & 31;
	const int      warp = tid >> 5;
	const int      wm   = warp % C::WARPS_M;
	const int      wn   = warp / C::WARPS_M;

	int total = 0;
	for (int s = t.seg_begin; s < t.seg_end; ++s)
		total += (args.segs[s].K + C::BK - 1) / C::BK;

	double acc[C::MI][C::NI][2];
#pragma unroll
	for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
		for (int ni = 0; ni < C::NI; ++ni)
			acc[mi][ni][0] = acc[mi][ni][1] = 0.0;

	// load cursor over the flattened (segment, k-chunk) sequence
	int     ls = t.seg_begin;
	int     lk = 0;
	GemmSeg cur {};
	if (ls < t.seg_end)
		cur = args.segs[ls];
	auto issue = [&](int stage) {
		load_stage<C>(As + stage * C::A_STAGE,
		              Bs + stage * C::B_STAGE,
		              args.A + cur.a_off,
		              cur.lda,
		              args.B + cur.b_off,
		              cur.ldb,
		              cur.K,
		              lk,
		              t,
		              tid);
		lk += C::BK;
		if (lk >= cur.K) {
			lk = 0;
			++ls;
			if (ls < t.seg_end)
				cur = args.segs[ls];
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
					dmma_8x8x4(acc[mi][ni][0], acc[mi][ni][1], af[mi], bf[ni]);
		}
	}
	cp_async_wait<0>();

	double* Cp = args.C + t.c_off;
#pragma unroll
	for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
		for (int ni = 0; ni < C::NI; ++ni)
#pragma unroll
			for (int h = 0; h < 2; ++h) {
				const int row = t.m0 + wm * C::WM + mi * 8 + (lane >> 2);
				const int col = t.n0 + wn * C::WN + ni * 8 + (lane & 3) * 2 + h;
				if (row < t.M && col < t.N)
					Cp[(long long)col * t.ldc + row] = acc[mi][ni][h];
			}
}

template <class C> cudaError_t launch_cfg(const GemmArgs& args, cudaStream_t stream)
{
	if (args.ntiles <= 0)
		return cudaSuccess;
	grouped_dgemm_kernel<C><<<args.ntiles, C::THREADS, C::SMEM, stream>>>(args);
	return cudaGetLastError();
}

using Cfg64 = TileCfg<64, 64, 16, 32, 32, 3>;
using Cfg32 = TileCfg<32, 32, 16, 16, 16, 3>;

template <class C> cudaError_t init_cfg()
{
	return cudaFuncSetAttribute(
	    grouped_dgemm_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(C::SMEM));
}

} // namespace

cudaError_t init_grouped_dgemm()
{
	cudaError_t e = init_cfg<Cfg64>();
	if (e == cudaSuccess)
		e = init_cfg<Cfg32>();
	return e;
}

cudaError_t launch_grouped_dgemm(const GemmArgs& args, int bm, int bn, cudaStream_t stream)
{
	if (bm == 64 && bn == 64)
		return launch_cfg<Cfg64>(args, stream);
	if (bm == 32 && bn == 32)
		return launch_cfg<Cfg32>(args, stream);
	return cudaErrorInvalidValue;
}

} // namespace dmrgpp
