// One persistent launch for a whole sector H*x: pass-1 tiles and (K-split)
// pass-2 tiles are pulled from one work queue by a fixed grid of CTAs.
//
// Ordering: every pass-1 item precedes every pass-2 item in the queue.  A
// pass-2 item first waits until all pass-1 tiles of the input patches its
// K-slice reads are complete (per-patch completion counters).  Pass-1 items
// never wait, and an item is only dequeued after all earlier items were
// dequeued by running CTAs, so the waits always end; they are still bounded
// in time (kWaitLimitNs); a wait that gives up raises the abort word, which
// ends every other wait, and the host-visible error word, and the launch
// runs to its end with an invalid result instead of hanging.
//
// Split-K: the parts of one output tile write partial tiles to their own
// slots; the part that arrives last sums the slots in slot order and stores
// the tile, so the result does not depend on arrival order (bitwise
// reproducible).
//
// Counters are returned to zero by the last CTA to leave, so consecutive
// launches (and CUDA-graph replays) need no memset.
//
// Per item the CTA pays a few global round trips (claim, descriptor,
// segments, the release of a finished pass-1 tile); they are overlapped
// with the previous item's stores (see the loop below).
//
// Group handles (independent sectors in one launch) may pass a per-sector
// active mask: the items of stopped sectors are claimed and dropped.
#include "kron_persistent.cuh"
#include "tile_dmma.cuh"

namespace dmrgpp {
namespace {

// Upper bound of one dependency wait (nanoseconds of %globaltimer).  A legal
// wait lasts at most one pass-1 tile (microseconds to a millisecond).
constexpr unsigned long long kWaitLimitNs = 200ull * 1000ull * 1000ull;

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
	unsigned long long t;
	asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
	return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
	unsigned v;
	asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
	return v;
}

template <class C>
__device__ __forceinline__ void
store_tile(const tile::Acc<C>& acc, double* Cp, int ldc, int m0, int n0, int M, int N)
{
#pragma unroll
	for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
		for (int ni = 0; ni < C::NI; ++ni)
#pragma unroll
			for (int h = 0; h < 2; ++h) {
				const int row = m0 + tile::acc_row<C>(mi);
				const int col = n0 + tile::acc_col<C>(ni, h);
				if (row < M && col < N)
					Cp[(long long)col * ldc + row] = acc.v[mi][ni][h];
			}
}

template <class C>
__global__ void __launch_bounds__(C::THREADS) kron_persistent_kernel(PersistentArgs a)
{
	extern __shared__ __align__(16) double smem[];
	__shared__ __align__(16) KronItem s_w[2];
	__shared__ __align__(16) GemmSeg  s_seg[2][kMaxItemSegs];
	__shared__ int                    s_it[2];
	__shared__ int                    s_last;
	const int                         tid  = threadIdx.x;
	const int                         warp = tid >> 5, lane = tid & 31;
	tile::Acc<C>                      acc;
	const double*                     X   = a.io ? a.io->x : a.x;
	double*                           Y   = a.io ? a.io->y : a.y;
	constexpr int                     kSegWords = int(sizeof(GemmSeg) / sizeof(int));
	constexpr int                     kItemVec  = int(sizeof(KronItem) / 16);
	static_assert(sizeof(KronItem) % 16 == 0, "descriptor copy");
	static_assert(kItemVec <= 32, "one warp loads a descriptor");

	// Work distribution: the first item of every CTA is its block index;
	// later items are claimed one at a time from a counter offset by the grid
	// size.  During a pass-1 item the next one is claimed only when its MMAs
	// are done, which keeps the remaining pass-1 items (which pass-2 items
	// wait on) from queueing behind busy CTAs; during a pass-2 item it is
	// claimed at the start, so the claim and the loads of its descriptor and
	// segments (by warp 0, into the other of two buffers) overlap the
	// dependency wait and the MMAs.  Items of stopped sectors of a group are
	// claimed and dropped here.
	auto fetch = [&](int buf, int it) { // warp 0
		for (;;) {
			if (it < a.n_items && a.sector_active && !a.sector_active[a.item_sector[it]]) {
				unsigned nx = 0;
				if (lane == 0)
					nx = atomicAdd(&a.work_counter[0], 1u);
				it = int(gridDim.x + __shfl_sync(0xffffffffu, nx, 0));
				continue;
			}
			break;
		}
		if (lane == 0)
			s_it[buf] = it;
		if (it >= a.n_items)
			return;
		if (lane < kItemVec)
			reinterpret_cast<int4*>(&s_w[buf])[lane] = reinterpret_cast<const int4*>(a.items + it)[lane];
		__syncwarp();
		const KronItem& w    = s_w[buf];
		const int       nseg = w.seg_end - w.seg_begin;
		if (nseg > 1) {
			const GemmSeg* gseg = (w.kind == 0 ? a.seg1 : a.pseg2) + w.seg_begin;
			for (int q = lane; q < nseg * kSegWords; q += 32)
				reinterpret_cast<int*>(s_seg[buf])[q] = reinterpret_cast<const int*>(gseg)[q];
		} else if (lane < kSegWords) {
			reinterpret_cast<int*>(s_seg[buf])[lane] = reinterpret_cast<const int*>(&w.seg0)[lane];
		}
	};
	auto claim_next = [&](int buf) { // warp 0
		unsigned nx = 0;
		if (lane == 0)
			nx = atomicAdd(&a.work_counter[0], 1u);
		fetch(buf, int(gridDim.x + __shfl_sync(0xffffffffu, nx, 0)));
	};

	if (warp == 0)
		fetch(0, int(blockIdx.x));
	__syncthreads();
	for (int cur = 0;; cur ^= 1) {
		const int it = s_it[cur];
		if (it >= a.n_items)
			break;
		const KronItem& w    = s_w[cur];
		const GemmSeg*  sg   = s_seg[cur];
		const int       nseg = w.seg_end - w.seg_begin;

		if (w.kind == 0) {
			tile::mma_tile<C>(acc, smem, a.ops, X, sg, 0, nseg, w.m0, w.n0, w.M, w.N);
			if (warp == 0)
				claim_next(cur ^ 1);
			store_tile<C>(acc, a.bx + w.c_off, w.ldc, w.m0, w.n0, w.M, w.N);
			__syncthreads(); // tile stored; next descriptor visible
			if (tid == 0) {
				__threadfence();
				atomicAdd(&a.done[w.producer], 1u);
			}
			continue;
		}
		// a pass-2 item blocks no other item: claim and fetch the next one
		// now, behind this item's dependency wait and MMAs
		if (warp == 0)
			claim_next(cur ^ 1);
		if (tid == 0) {
			int last_dep = -1;
			for (int s = 0; s < nseg; ++s) {
				const int j = sg[s].dep;
				if (j == last_dep)
					continue;
				last_dep = j;
				const unsigned target = unsigned(a.n1_of_j[j] + (j == 0 ? a.test_extra_wait : 0));
				const unsigned long long t0 = globaltimer_ns();
				while (ld_acquire(&a.done[j]) < target) {
					if (ld_acquire(&a.work_counter[2]) != 0u)
						break; // another wait already gave up
					if (globaltimer_ns() - t0 > kWaitLimitNs) {
						atomicExch(&a.work_counter[2], 1u);
						*reinterpret_cast<volatile int*>(a.error) = 1;
						__threadfence_system();
						break;
					}
					__nanosleep(128);
				}
			}
		}
		__syncthreads();
		tile::mma_tile<C>(acc, smem, a.bx, a.ops, sg, 0, nseg, w.m0, w.n0, w.M, w.N);
		if (w.kind == 1) {
			store_tile<C>(acc, Y + w.c_off, w.ldc, w.m0, w.n0, w.M, w.N);
			__syncthreads(); // next descriptor visible
			continue;
		}
		// split part: partial tile to its slot, the last part reduces
		constexpr int TE   = C::BM * C::BN;
		double*       part = a.partial + (long long)(w.slot + w.part) * TE;
#pragma unroll
		for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
			for (int ni = 0; ni < C::NI; ++ni)
#pragma unroll
				for (int h = 0; h < 2; ++h)
					part[tile::acc_col<C>(ni, h) * C::BM + tile::acc_row<C>(mi)] = acc.v[mi][ni][h];
		__syncthreads();
		if (tid == 0) {
			__threadfence();
			const unsigned old = atomicAdd(&a.arrive[w.tile], 1u);
			s_last             = (old == unsigned(w.nsplit - 1));
			if (s_last)
				__threadfence();
		}
		__syncthreads();
		if (s_last) {
			const double* slots = a.partial + (long long)w.slot * TE;
			double*       Cp    = Y + w.c_off;
#pragma unroll
			for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
				for (int ni = 0; ni < C::NI; ++ni)
#pragma unroll
					for (int h = 0; h < 2; ++h) {
						const int r   = tile::acc_row<C>(mi);
						const int c   = tile::acc_col<C>(ni, h);
						const int e   = c * C::BM + r;
						double    sum = __ldcg(slots + e);
						for (int p = 1; p < w.nsplit; ++p)
							sum += __ldcg(slots + (long long)p * TE + e);
						const int row = w.m0 + r, col = w.n0 + c;
						if (row < w.M && col < w.N)
							Cp[(long long)col * w.ldc + row] = sum;
					}
		}
		__syncthreads(); // s_last read by everyone before the next part may set it
	}

	// the last CTA out returns every counter to zero for the next launch
	if (tid == 0) {
		__threadfence();
		const unsigned old = atomicAdd(&a.work_counter[1], 1u);
		if (old == gridDim.x - 1) {
			for (int j = 0; j < a.np; ++j)
				a.done[j] = 0u;
			for (int t = 0; t < a.n_split_tiles; ++t)
				a.arrive[t] = 0u;
			a.work_counter[0] = 0u;
			a.work_counter[2] = 0u;
			__threadfence();
			a.work_counter[1] = 0u;
		}
	}
}

// Tile configurations a handle can run (kron_persistent.cuh, KronTileCfg).
using PCfg0 = tile::Cfg<32, 32, 16, 16, 16, 4>;
using PCfg1 = tile::Cfg<32, 32, 32, 16, 16, 3>;
using PCfg2 = tile::Cfg<64, 64, 16, 32, 32, 3>;
using PCfg3 = tile::Cfg<64, 64, 32, 32, 32, 3>;
using PCfg4 = tile::Cfg<32, 32, 32, 16, 16, 4>;
using PCfg5 = tile::Cfg<32, 32, 64, 16, 16, 3>;

template <class C> cudaError_t init_one(int* blocks_per_sm)
{
	cudaError_t e = cudaFuncSetAttribute(kron_persistent_kernel<C>,
	                                     cudaFuncAttributeMaxDynamicSharedMemorySize, int(C::SMEM));
	if (e != cudaSuccess)
		return e;
	return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kron_persistent_kernel<C>,
	                                                     C::THREADS, C::SMEM);
}

template <class C> void describe(int* tile, int* bk)
{
	*tile = C::BM;
	*bk   = C::BK;
}

} // namespace

cudaError_t persistent_config(int cfg, int* grid, int* tile, int* bk)
{
	int         dev = 0, sms = 0, per_sm = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e == cudaSuccess)
		e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	if (e != cudaSuccess)
		return e;
	switch (cfg) {
	case 0: e = init_one<PCfg0>(&per_sm); describe<PCfg0>(tile, bk); break;
	case 1: e = init_one<PCfg1>(&per_sm); describe<PCfg1>(tile, bk); break;
	case 2: e = init_one<PCfg2>(&per_sm); describe<PCfg2>(tile, bk); break;
	case 3: e = init_one<PCfg3>(&per_sm); describe<PCfg3>(tile, bk); break;
	case 4: e = init_one<PCfg4>(&per_sm); describe<PCfg4>(tile, bk); break;
	case 5: e = init_one<PCfg5>(&per_sm); describe<PCfg5>(tile, bk); break;
	default: return cudaErrorInvalidValue;
	}
	if (e != cudaSuccess)
		return e;
	*grid = sms * (per_sm > 0 ? per_sm : 1);
	return cudaSuccess;
}

cudaError_t launch_persistent(const PersistentArgs& a, int cfg, int grid, cudaStream_t stream)
{
	if (a.n_items <= 0)
		return cudaSuccess;
	const int g = grid < a.n_items ? grid : a.n_items;
	switch (cfg) {
	case 0: kron_persistent_kernel<PCfg0><<<g, PCfg0::THREADS, PCfg0::SMEM, stream>>>(a); break;
	case 1: kron_persistent_kernel<PCfg1><<<g, PCfg1::THREADS, PCfg1::SMEM, stream>>>(a); break;
	case 2: kron_persistent_kernel<PCfg2><<<g, PCfg2::THREADS, PCfg2::SMEM, stream>>>(a); break;
	case 3: kron_persistent_kernel<PCfg3><<<g, PCfg3::THREADS, PCfg3::SMEM, stream>>>(a); break;
	case 4: kron_persistent_kernel<PCfg4><<<g, PCfg4::THREADS, PCfg4::SMEM, stream>>>(a); break;
	case 5: kron_persistent_kernel<PCfg5><<<g, PCfg5::THREADS, PCfg5::SMEM, stream>>>(a); break;
	default: return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

} // namespace dmrgpp
