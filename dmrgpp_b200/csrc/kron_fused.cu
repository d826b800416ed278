// Fused FP64 H*x for sectors of small patches: one CTA computes both passes
// of (part of) one output tile, so no pass-1 result crosses between CTAs and
// nothing waits on another CTA's work.
//
// Output tile [m0, m0+BM) x [n0, n0+BN) of Y_i.  Its work is a list of units
// (kron_plan.h, FusedUnit), one per contributing (j,k) and CW-column chunk
// c of X_j:
//     T = B_k(i,j)[rows, :] * X_j[:, c]          (BM x CW, in shared memory)
//     acc += T * A_k(i,j)[cols, c]^T             (BM x BN, in registers)
// The chunks of X_j's columns are the contraction of the second product, so
// splitting a tile's units over several CTAs repeats no work.  The parts of
// one tile run in one thread-block cluster; each writes its partial tile to
// its own shared memory, and after a cluster barrier part p sums slice p of
// the tile over all parts in part order (distributed shared memory reads) and
// stores it, so the result is bitwise reproducible and no partial tile goes
// through global memory.  A cluster may hold several tiles (packed whole on
// the host); empty slots only take part in the two cluster barriers.
//
// Every CTA reaches both cluster barriers whatever its work (inactive
// sectors, empty slots), and there is no other wait: the launch cannot
// block on a condition that never comes.
//
// Inner products on the FP64 tensor pipe (mma.sync m8n8k4, as in the
// persistent kernel), operands global -> shared by 8-byte cp.async with
// zero fill, one STAGES-deep ring shared by both products.
#include "kron_fused.cuh"
#include "tile_dmma.cuh"

#include <cooperative_groups.h>

namespace dmrgpp {
namespace {

namespace cg = cooperative_groups;

template <int BM_, int CW_, int BN_, int BK_, int STAGES_, int WARPS_, int W1M_, int W2M_, int SK1_ = 1>
struct FCfg {
	static constexpr int BM = BM_, CW = CW_, BN = BN_, BK = BK_, STAGES = STAGES_;
	static constexpr int WARPS = WARPS_, THREADS = 32 * WARPS_;
	// first product T (BM x CW): W1M x W1N warps of WM1 x WN1, or (SK1 > 1)
	// every warp the whole T over every SK1-th k-step of four, the SK1 partial
	// T tiles summed in shared memory; second product (BM x BN): W2M x W2N
	// warps of WM2 x WN2
	static constexpr int SK1 = SK1_;
	static constexpr int W1M = W1M_, W1N = SK1 > 1 ? 1 : WARPS / W1M_, WM1 = BM / W1M_, WN1 = CW / W1N;
	static constexpr int W2M = W2M_, W2N = WARPS / W2M_, WM2 = BM / W2M_, WN2 = BN / W2N;
	static constexpr int MI1 = WM1 / 8, NI1 = WN1 / 8;
	static constexpr int MI2 = WM2 / 8, NI2 = WN2 / 8;
	// shared memory, in doubles: ring stages of an A tile [k][m] (rows of
	// B_k(i,j)) and a B tile [n][k] (columns of X_j, or of A^T), the T tile
	// [k][m], and the partial tile [col][row] (over the ring, after it)
	static constexpr int LDA     = BM + 4;
	static constexpr int LDB     = BK + 4;
	static constexpr int NB      = BN > CW ? BN : CW;
	static constexpr int A_STAGE = BK * LDA;
	static constexpr int STAGE   = A_STAGE + NB * LDB;
	static constexpr int RING    = STAGES * STAGE;
	static constexpr int LDP     = BM + 1;
	static constexpr int P_ELEMS = BN * LDP;
	static constexpr int T_OFF   = RING > P_ELEMS ? RING : P_ELEMS;
	static constexpr int T_ELEMS = CW * LDA;
	static constexpr size_t SMEM = size_t(T_OFF + SK1 * T_ELEMS) * sizeof(double);
	static_assert(WM1 % 8 == 0 && WN1 % 8 == 0 && WM2 % 8 == 0 && WN2 % 8 == 0, "warp tiles");
	static_assert(W1M * W1N * SK1 == WARPS && W2M * W2N == WARPS, "warp grid");
	static_assert(SK1 == 1 || BK / 4 == SK1, "one k-step of four per warp and stage");
	static_assert(BK % 4 == 0, "k step");
	static_assert((BM * BK) % THREADS == 0 && (CW * BK) % THREADS == 0 && (BN * BK) % THREADS == 0,
	              "load split");
};

// Position in the step sequence of an item: unit u, product (0: T = B X,
// 1: acc += T A^T) and offset k0 in that product's contraction.
struct Cursor {
	int       u, phase, k0;
	FusedUnit d;
};

template <class C> __device__ __forceinline__ void cursor_at(Cursor& c, const FusedUnit* units, int u, int u_end)
{
	c.u     = u;
	c.phase = 0;
	c.k0    = 0;
	if (u < u_end)
		c.d = units[u];
}

template <class C> __device__ __forceinline__ void cursor_next(Cursor& c, const FusedUnit* units, int u_end)
{
	c.k0 += C::BK;
	const int K = c.phase == 0 ? c.d.rj : c.d.cw;
	if (c.k0 < K)
		return;
	c.k0 = 0;
	if (c.phase == 0) {
		c.phase = 1;
		return;
	}
	c.phase = 0;
	if (++c.u < u_end)
		c.d = units[c.u];
}

// Enqueues the loads of step c into ring stage `stage`.
template <class C>
__device__ __forceinline__ void issue(const Cursor& c, double* stage, const double* ops, const double* X,
                                      int M, int N, int m0, int n0, int tid)
{
	double* As = stage;
	double* Bs = stage + C::A_STAGE;
	if (c.phase == 0) {
		const double* b  = ops + c.d.b_off;
		const double* xj = X + c.d.x_off;
#pragma unroll
		for (int e = 0; e < C::BM * C::BK / C::THREADS; ++e) {
			const int  idx = tid + e * C::THREADS;
			const int  m = idx % C::BM, kk = idx / C::BM;
			const int  gk = c.k0 + kk;
			const bool p  = m0 + m < M && gk < c.d.rj;
			tile::cp_async_8(tile::smem_u32(As + kk * C::LDA + m),
			                 p ? b + (long long)gk * c.d.ldb + m0 + m : b, p);
		}
#pragma unroll
		for (int e = 0; e < C::CW * C::BK / C::THREADS; ++e) {
			const int  idx = tid + e * C::THREADS;
			const int  kk = idx % C::BK, n = idx / C::BK;
			const int  gk = c.k0 + kk;
			const bool p  = n < c.d.cw && gk < c.d.rj;
			tile::cp_async_8(tile::smem_u32(Bs + n * C::LDB + kk),
			                 p ? xj + (long long)n * c.d.rj + gk : xj, p);
		}
	} else {
		const double* at = ops + c.d.at_off;
#pragma unroll
		for (int e = 0; e < C::BN * C::BK / C::THREADS; ++e) {
			const int  idx = tid + e * C::THREADS;
			const int  kk = idx % C::BK, n = idx / C::BK;
			const int  gk = c.k0 + kk;
			const bool p  = n0 + n < N && gk < c.d.cw;
			tile::cp_async_8(tile::smem_u32(Bs + n * C::LDB + kk),
			                 p ? at + (long long)(n0 + n) * c.d.lj + gk : at, p);
		}
	}
}

// One item (the CTA's part of one cluster slot), ending with the cluster's
// reduction of every tile of the slot.
template <class C>
__device__ __forceinline__ void fused_slot(const FusedArgs& a, const FusedItem it, double* smem,
                                           cg::cluster_group& cluster)
{
	const int         tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const bool        active = it.nparts > 0 && (!a.sector_active || a.sector_active[it.sector]);
	const double*     X      = a.io ? a.io->x : a.x;
	double*           Y      = a.io ? a.io->y : a.y;
	double*           Ts     = smem + C::T_OFF;
	const int         Mt     = active ? min(C::BM, it.M - it.m0) : 0; // valid rows of the tile
	const int         Nt     = active ? min(C::BN, it.N - it.n0) : 0; // valid columns

	double acc[C::MI2][C::NI2][2];
#pragma unroll
	for (int mi = 0; mi < C::MI2; ++mi)
#pragma unroll
		for (int ni = 0; ni < C::NI2; ++ni)
			acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
	double t1[C::MI1][C::NI1][2];

	const int u_end = active ? it.u_end : it.u_begin;
	// warp tiles of the two products (with the first product split along its
	// contraction every warp covers the whole T tile)
	const int wm1 = C::SK1 > 1 ? 0 : warp / C::W1N, wn1 = C::SK1 > 1 ? 0 : warp % C::W1N;
	const int wm2 = warp / C::W2N, wn2 = warp % C::W2N;
	Cursor    ld, cs;
	cursor_at<C>(ld, a.units, it.u_begin, u_end);
	cursor_at<C>(cs, a.units, it.u_begin, u_end);
#pragma unroll
	for (int s = 0; s < C::STAGES - 1; ++s) {
		if (ld.u < u_end) {
			issue<C>(ld, smem + s * C::STAGE, a.ops, X, it.M, it.N, it.m0, it.n0, tid);
			cursor_next<C>(ld, a.units, u_end);
		}
		tile::cp_async_commit();
	}
	for (int step = 0; cs.u < u_end; ++step) {
		tile::cp_async_wait<C::STAGES - 2>();
		__syncthreads();
		if (ld.u < u_end) {
			issue<C>(ld, smem + ((step + C::STAGES - 1) % C::STAGES) * C::STAGE, a.ops, X, it.M, it.N,
			         it.m0, it.n0, tid);
			cursor_next<C>(ld, a.units, u_end);
		}
		tile::cp_async_commit();
		if (C::SK1 > 1 && cs.phase == 1 && cs.k0 == 0) { // the partial T tiles, summed in warp order
			for (int e = tid; e < C::T_ELEMS; e += C::THREADS) {
				double t = Ts[e];
#pragma unroll
				for (int w = 1; w < C::SK1; ++w)
					t += Ts[w * C::T_ELEMS + e];
				Ts[e] = t;
			}
			__syncthreads();
		}
		const double* As   = smem + (step % C::STAGES) * C::STAGE;
		const double* Bs   = As + C::A_STAGE;
		const int     K    = cs.phase == 0 ? cs.d.rj : cs.d.cw;
		const int     kmax = min(C::BK, K - cs.k0);
		if (cs.phase == 0) {
			if (cs.k0 == 0) {
#pragma unroll
				for (int mi = 0; mi < C::MI1; ++mi)
#pragma unroll
					for (int ni = 0; ni < C::NI1; ++ni)
						t1[mi][ni][0] = t1[mi][ni][1] = 0.0;
			}
			const double* as = As + wm1 * C::WM1 + (lane >> 2);
			const double* bs = Bs + (wn1 * C::WN1 + (lane >> 2)) * C::LDB;
#pragma unroll
			for (int ks = 0; ks < C::BK; ks += 4) {
				if (ks < kmax && (C::SK1 == 1 || ks / 4 == warp)) {
					double af[C::MI1], bf[C::NI1];
#pragma unroll
					for (int mi = 0; mi < C::MI1; ++mi)
						af[mi] = as[(ks + (lane & 3)) * C::LDA + mi * 8];
#pragma unroll
					for (int ni = 0; ni < C::NI1; ++ni)
						bf[ni] = bs[ni * 8 * C::LDB + ks + (lane & 3)];
#pragma unroll
					for (int mi = 0; mi < C::MI1; ++mi)
#pragma unroll
						for (int ni = 0; ni < C::NI1; ++ni)
							if (wm1 * C::WM1 + mi * 8 < Mt && wn1 * C::WN1 + ni * 8 < cs.d.cw)
								tile::dmma_8x8x4(t1[mi][ni][0], t1[mi][ni][1], af[mi], bf[ni]);
				}
			}
			if (cs.k0 + C::BK >= K) { // T complete: to shared memory as [k][m]
#pragma unroll
				for (int mi = 0; mi < C::MI1; ++mi)
#pragma unroll
					for (int ni = 0; ni < C::NI1; ++ni)
#pragma unroll
						for (int h = 0; h < 2; ++h) {
							const int row = wm1 * C::WM1 + mi * 8 + (lane >> 2);
							const int col = wn1 * C::WN1 + ni * 8 + (lane & 3) * 2 + h;
							Ts[(C::SK1 > 1 ? warp * C::T_ELEMS : 0) + col * C::LDA + row] = t1[mi][ni][h];
						}
			}
		} else {
			const double* as = Ts + cs.k0 * C::LDA + wm2 * C::WM2 + (lane >> 2);
			const double* bs = Bs + (wn2 * C::WN2 + (lane >> 2)) * C::LDB;
#pragma unroll
			for (int ks = 0; ks < C::BK; ks += 4) {
				if (ks < kmax) {
					double af[C::MI2], bf[C::NI2];
#pragma unroll
					for (int mi = 0; mi < C::MI2; ++mi)
						af[mi] = as[(ks + (lane & 3)) * C::LDA + mi * 8];
#pragma unroll
					for (int ni = 0; ni < C::NI2; ++ni)
						bf[ni] = bs[ni * 8 * C::LDB + ks + (lane & 3)];
#pragma unroll
					for (int mi = 0; mi < C::MI2; ++mi)
#pragma unroll
						for (int ni = 0; ni < C::NI2; ++ni)
							if (wm2 * C::WM2 + mi * 8 < Mt && wn2 * C::WN2 + ni * 8 < Nt)
								tile::dmma_8x8x4(acc[mi][ni][0], acc[mi][ni][1], af[mi], bf[ni]);
				}
			}
		}
		cursor_next<C>(cs, a.units, u_end);
	}
	tile::cp_async_wait<0>();
	__syncthreads(); // ring free: the partial tile goes over it

	double* Pt = smem;
#pragma unroll
	for (int mi = 0; mi < C::MI2; ++mi)
#pragma unroll
		for (int ni = 0; ni < C::NI2; ++ni)
#pragma unroll
			for (int h = 0; h < 2; ++h) {
				const int row = wm2 * C::WM2 + mi * 8 + (lane >> 2);
				const int col = wn2 * C::WN2 + ni * 8 + (lane & 3) * 2 + h;
				Pt[col * C::LDP + row] = acc[mi][ni][h];
			}
	cluster.sync(); // every part's partial tile is visible to the cluster

	if (active) {
		const long long E  = (long long)Mt * Nt;
		const long long e0 = E * it.part / it.nparts, e1 = E * (it.part + 1) / it.nparts;
		double*         Yt = Y + it.y_off + (long long)it.n0 * it.M + it.m0;
		for (long long e = e0 + tid; e < e1; e += C::THREADS) {
			const int     col = int(e / Mt), row = int(e - (long long)col * Mt);
			const int     off = col * C::LDP + row;
			double        sum = cluster.map_shared_rank(Pt, it.rank0)[off];
			for (int q = 1; q < it.nparts; ++q)
				sum += cluster.map_shared_rank(Pt, it.rank0 + q)[off];
			Yt[(long long)col * it.M + row] = sum;
		}
	}
	cluster.sync(); // no CTA goes on (or leaves) while another may still read its partial
}

template <class C>
__global__ void __launch_bounds__(C::THREADS, C::WARPS == 4 ? 2 : 1) kron_fused_kernel(FusedArgs a)
{
	extern __shared__ __align__(16) double smem[];
	cg::cluster_group cluster = cg::this_cluster();
	const int         S       = int(cluster.num_blocks());
	const int         nslots  = a.n_items / S;
	// the clusters of the grid walk the cluster slots of the schedule; every
	// CTA of a cluster takes the same slots, so all meet the same barriers
	for (int slot = int(blockIdx.x) / S; slot < nslots; slot += int(gridDim.x) / S)
		fused_slot<C>(a, a.items[slot * S + int(cluster.block_rank())], smem, cluster);
}


// BM x CW x BN tiles, k-steps of 16, three stages, four warps (two CTAs per
// SM: sixteen independent accumulator chains per warp keep the FP64 pipe
// busy).  Measured alternatives, not kept (microbench sector): eight warps
// at one CTA per SM (clusters of 8 then occupy 120 of 148 SMs), 16-row tiles
// (too few accumulator chains per warp), 32-column units with the first
// product's contraction split over the warps, k-steps of 32.
using F0 = FCfg<32, 64, 128, 16, 3, 4, 1, 1, 1>;

template <class C> cudaLaunchConfig_t launch_config(int clusters, int cluster, cudaStream_t stream,
                                                    cudaLaunchAttribute* attr)
{
	cudaLaunchConfig_t cfg {};
	cfg.gridDim          = dim3(unsigned(clusters * cluster), 1, 1);
	cfg.blockDim         = dim3(C::THREADS, 1, 1);
	cfg.dynamicSmemBytes = C::SMEM;
	cfg.stream           = stream;
	attr[0].id               = cudaLaunchAttributeClusterDimension;
	attr[0].val.clusterDim.x = unsigned(cluster);
	attr[0].val.clusterDim.y = 1;
	attr[0].val.clusterDim.z = 1;
	cfg.attrs                = attr;
	cfg.numAttrs             = 1;
	return cfg;
}

template <class C> cudaError_t max_clusters(int cluster, int* out)
{
	cudaLaunchAttribute attr[1];
	cudaLaunchConfig_t  cfg = launch_config<C>(1, cluster, nullptr, attr);
	return cudaOccupancyMaxActiveClusters(out, kron_fused_kernel<C>, &cfg);
}

template <class C> cudaError_t init_one(int cluster, int* clusters)
{
	cudaError_t e = cudaFuncSetAttribute(kron_fused_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                     int(C::SMEM));
	if (e == cudaSuccess && cluster > 8)
		e = cudaFuncSetAttribute(kron_fused_kernel<C>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
	if (e == cudaSuccess)
		e = max_clusters<C>(cluster, clusters);
	return e;
}

template <class C> cudaError_t launch_one(const FusedArgs& a, int cluster, cudaStream_t stream)
{
	const int          slots    = a.n_items / cluster;
	const int          clusters = a.max_clusters > 0 && a.max_clusters < slots ? a.max_clusters : slots;
	cudaLaunchAttribute attr[1];
	cudaLaunchConfig_t  cfg = launch_config<C>(clusters, cluster, stream, attr);
	return cudaLaunchKernelEx(&cfg, kron_fused_kernel<C>, a);
}

} // namespace

FusedShape fused_shape(int fcfg)
{
	static const FusedShape shapes[kNumFusedCfgs] = { { 32, 64, 128, 8 }, { 32, 64, 128, 16 } };
	return shapes[(fcfg >= 0 && fcfg < kNumFusedCfgs) ? fcfg : 0];
}

cudaError_t fused_init(int fcfg, int* clusters)
{
	if (fcfg < 0 || fcfg >= kNumFusedCfgs)
		return cudaErrorInvalidValue;
	const FusedShape s = fused_shape(fcfg);
	return init_one<F0>(s.cluster, clusters);
}

cudaError_t launch_fused(const FusedArgs& a, int fcfg, cudaStream_t stream)
{
	if (fcfg < 0 || fcfg >= kNumFusedCfgs)
		return cudaErrorInvalidValue;
	if (a.n_items <= 0)
		return cudaSuccess;
	const FusedShape s = fused_shape(fcfg);
	if (a.n_items % s.cluster != 0)
		return cudaErrorInvalidValue;
	return launch_one<F0>(a, s.cluster, stream);
}

} // namespace dmrgpp
