// Mixed-precision grouped GEMM on the 5th-generation tensor cores (tcgen05).
//
// TF32x3: each FP64 operand is carried as two TF32 parts, a = a_hi + a_lo, and
// one tile accumulates a_hi*b_hi + a_hi*b_lo + a_lo*b_hi in FP32 in tensor
// memory (the a_lo*b_lo term is below the FP32 accumulation error).
//
// Persistent, warp-specialised CTAs (at most one per SM), each walking its
// own run of the tile list of one grouped pass (kron_plan.h, MixedPlan;
// runs balanced on the host by balance_tiles):
//   warp 0, one thread: producer.  For every 32-wide k-chunk of every
//     K-segment of its tiles it waits until the ring stage is free, arms the
//     stage's mbarrier with the byte count and issues four tiled TMA loads
//     (cp.async.bulk.tensor.2d, completion counted on the mbarrier): the hi
//     and lo parts of the A tile (128 rows) and of the B tile (BN rows).
//     Every operand buffer is a 2-D tensor [row][32 values] (kron_plan.h;
//     the tensor maps are kernel parameters); the TMA unit writes the tile
//     in the 128-byte-swizzled K-major layout tcgen05.mma reads.  The x
//     coordinate is always 0.
//   warp 1, one thread: MMA issuer.  Per chunk it waits for the stage's
//     bytes, issues 3 x 4 MMAs (M = 128, N = BN, K = 8) into the tile's TMEM
//     accumulator and commits them to the stage's "empty" mbarrier; after
//     the tile's last chunk it commits to the accumulator's "full" mbarrier.
//     Two accumulators (2 x BN TMEM columns) alternate between tiles, so one
//     tile's epilogue overlaps the next tile's loads and MMAs.
//   warps 2-5: epilogue.  Warp w reads TMEM lanes 32(w % 4) .. +31 (tile
//     rows) with tcgen05.ld and either splits the result into the hi/lo
//     chunked layout of the next pass (pass 1: BX, the A operand of pass 2)
//     or widens it to FP64 (pass 2: y), then frees the accumulator.  In
//     pass 1 a thread's 32 values of one chunk are one 128-byte row of BX;
//     the warp writes its 32 rows into its own shared-memory staging tile
//     in the 128-byte-swizzled layout (no bank conflicts) and one lane
//     stores the tile with a tiled TMA store (a row-per-lane global store
//     would touch 32 lines per instruction).
//
// Every mbarrier wait is bounded in time and also ends when another role
// has given up (shared abort flag); a wait that gives up sets the error
// word.  Before the CTA exits, the producer waits (bounded) for its last
// copies and the MMA thread for its last MMAs, and TMEM is freed.
#include "tc_common.cuh"
#include "tc_gemm.cuh"

#include <cstdint>

namespace dmrgpp {
namespace {

using namespace tc;

constexpr int                kBM        = 128;
constexpr int                kBK        = 32; // TF32 elements = 128 bytes per row per chunk
constexpr int                kTcThreads = 192; // producer, MMA, 4 epilogue warps

// tiled TMA load of box (0, row) of a 2-D tensor into this CTA's shared
// memory, completion counted in bytes on the mbarrier
__device__ __forceinline__ void tma_load_2d(unsigned dst, const CUtensorMap* map, int row, unsigned mbar)
{
	asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
	             "[%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
	             "l"(reinterpret_cast<unsigned long long>(map)), "r"(0), "r"(row), "r"(mbar)
	             : "memory");
}

// tiled TMA store of a 32-row box from this CTA's shared memory to rows
// row .. row+31 of a 2-D tensor (bulk async-group of the issuing thread)
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, unsigned src, int row)
{
	asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(
	                 reinterpret_cast<unsigned long long>(map)),
	             "r"(0), "r"(row), "r"(src)
	             : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }

// the issuing thread's bulk stores have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }

// the issuing thread's bulk stores are complete (written to global memory)
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

// generic-proxy writes to shared memory become visible to the TMA unit
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void st_shared_v4(unsigned addr, float a, float b, float c, float d)
{
	asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};\n" ::"r"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
	             : "memory");
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

__device__ __forceinline__ int tile_chunks(const TcArgs& a, const GemmTile& t)
{
	int n = 0;
	for (int s = t.seg_begin; s < t.seg_end; ++s)
		n += a.segs[s].K / kBK;
	return n;
}

__device__ __forceinline__ void give_up(volatile int* abort, int* error)
{
	*abort = 1;
	atomicExch(error, 2);
}

// Tiles of a stopped sector are skipped by all three roles alike (the flags
// do not change during a launch), so the stage and accumulator phases stay
// in step; a pass-2 tile and all its K-split parts share one sector.
__device__ __forceinline__ bool skip_tile(const TcArgs& a, int ti)
{
	return a.sector_active && !a.sector_active[a.tile_sector[ti]];
}

// ---------------------------------------------------------------- producer
template <int BN, int STAGES>
__device__ void producer(const TcArgs& a, unsigned base, unsigned full0, unsigned empty0,
                         volatile int* abort)
{
	using L    = TcLayout<BN>;
	unsigned g = 0; // chunks issued
	bool     ok = true;
	// a tiled load moves its whole box (rows past the buffer arrive as 0)
	constexpr unsigned kStageTx = 2u * unsigned(L::A_BYTES + L::B_BYTES);
	for (int ti = a.starts[blockIdx.x]; ti < a.starts[blockIdx.x + 1] && ok; ++ti) {
		if (skip_tile(a, ti))
			continue;
		const GemmTile t = a.tiles[ti];
		for (int s = t.seg_begin; s < t.seg_end && ok; ++s) {
			const GemmSeg sg   = a.segs[s];
			const int     nk   = sg.K / kBK;
			const int     arow = int(sg.a_off) + t.m0; // buffer row of chunk 0
			const int     brow = int(sg.b_off) + t.n0;
			for (int c = 0; c < nk; ++c) {
				const unsigned st = g % STAGES;
				if (g >= STAGES && !mbar_wait(empty0 + 8 * st, ((g / STAGES) - 1) & 1, abort)) {
					ok = false;
					break;
				}
				const unsigned fb = full0 + 8 * st;
				const unsigned sa = base + st * unsigned(L::STAGE_BYTES);
				if (a.test_unarmed && blockIdx.x == 0 && g == 0) {
					// test hook: chunk 0 of CTA 0 is never armed nor filled, so
					// the MMA thread's bounded wait on it runs out of time
					++g;
					continue;
				}
				mbar_expect_tx(fb, kStageTx);
				const int ya = arow + c * sg.lda, yb = brow + c * sg.ldb;
				tma_load_2d(sa, &a.A_hi, ya, fb);
				tma_load_2d(sa + L::A_BYTES, &a.A_lo, ya, fb);
				tma_load_2d(sa + 2 * L::A_BYTES, &a.B_hi, yb, fb);
				tma_load_2d(sa + 2 * L::A_BYTES + L::B_BYTES, &a.B_lo, yb, fb);
				++g;
			}
		}
	}
	if (!ok)
		give_up(abort, a.error);
	// the latest phase of every stage still written to must have landed
	// before the CTA may exit (a stage the test hook left unarmed never
	// completes; its bounded wait just runs out)
	for (unsigned q = g > STAGES ? g - STAGES : 0; q < g; ++q)
		mbar_wait(full0 + 8 * (q % STAGES), (q / STAGES) & 1, nullptr);
}

// ---------------------------------------------------------------- MMA issuer
template <int BN, int STAGES>
__device__ void mma_issuer(const TcArgs& a, unsigned base, unsigned tmem, unsigned full0,
                           unsigned empty0, unsigned accf0, unsigned acce0, unsigned drain,
                           volatile int* abort)
{
	using L               = TcLayout<BN>;
	const unsigned idesc  = idesc_tf32<BN>();
	unsigned       g      = 0; // chunks consumed
	unsigned       tc     = 0; // tiles accumulated
	bool           ok     = true;
	bool           issued = false;
	for (int ti = a.starts[blockIdx.x]; ti < a.starts[blockIdx.x + 1] && ok; ++ti) {
		if (skip_tile(a, ti))
			continue;
		const GemmTile t     = a.tiles[ti];
		const int      total = tile_chunks(a, t);
		if (total == 0)
			continue;
		const unsigned b = tc & 1;
		if (tc >= 2 && !mbar_wait(acce0 + 8 * b, ((tc >> 1) - 1) & 1, abort)) {
			ok = false;
			break;
		}
		tc_fence_after();
		const unsigned d = tmem + b * unsigned(BN);
		for (int q = 0; q < total; ++q) {
			const unsigned st = g % STAGES;
			if (!mbar_wait(full0 + 8 * st, (g / STAGES) & 1, abort)) {
				ok = false;
				break;
			}
			tc_fence_after();
			const unsigned sa  = base + st * unsigned(L::STAGE_BYTES);
			const unsigned ahi = sa, alo = sa + L::A_BYTES;
			const unsigned bhi = sa + 2 * L::A_BYTES, blo = bhi + L::B_BYTES;
#pragma unroll
			for (int ks = 0; ks < kBK / 8; ++ks) {
				const unsigned kb = unsigned(ks * 32); // 8 TF32 = 32 bytes along K
				mma_tf32(d, smem_desc(ahi + kb), smem_desc(bhi + kb), idesc, (q | ks) != 0);
				mma_tf32(d, smem_desc(ahi + kb), smem_desc(blo + kb), idesc, 1u);
				mma_tf32(d, smem_desc(alo + kb), smem_desc(bhi + kb), idesc, 1u);
			}
			mma_commit(empty0 + 8 * st); // frees the stage once these MMAs are done
			issued = true;
			++g;
		}
		if (!ok)
			break;
		mma_commit(accf0 + 8 * b);
		++tc;
	}
	if (!ok)
		give_up(abort, a.error);
	// every MMA this thread issued must be complete before TMEM is freed
	if (issued) {
		mma_commit(drain);
		if (!mbar_wait(drain, 0, nullptr))
			give_up(abort, a.error);
	}
}

// ---------------------------------------------------------------- epilogue
template <int BN, bool PASS1>
__device__ __forceinline__ void store_chunk(const TcArgs& a, const GemmTile& t, int grow, int c0,
                                            const float (&v)[32])
{
	const int col0 = t.n0 + c0;
	if (grow >= t.M || col0 >= t.N)
		return;
	if (PASS1) {
		// one 128-byte row of chunk col0 / 32 of BX_j (hi and lo); columns
		// past N are the K padding of pass 2 and must be zero
		const long long o  = t.c_off + (long long)(col0 >> 5) * t.ldc * kBK + (long long)grow * kBK;
		// rows of one chunk are 128 bytes apart: a warp stores 4 KB contiguously
		float*          hi = a.C_hi + o;
		float*          lo = a.C_lo + o;
#pragma unroll
		for (int q = 0; q < 8; ++q) {
			float hv[4], lv[4];
#pragma unroll
			for (int e = 0; e < 4; ++e) {
				const float x = (col0 + 4 * q + e < t.N) ? v[4 * q + e] : 0.f;
				hv[e]         = tf32_rna(x);
				lv[e]         = tf32_rna(x - hv[e]);
			}
			*reinterpret_cast<float4*>(hi + 4 * q) = make_float4(hv[0], hv[1], hv[2], hv[3]);
			*reinterpret_cast<float4*>(lo + 4 * q) = make_float4(lv[0], lv[1], lv[2], lv[3]);
		}
	} else {
		double* y = (a.io ? a.io->y : a.Cd) + t.c_off;
#pragma unroll
		for (int i = 0; i < 32; ++i) {
			const int gcol = col0 + i;
			if (gcol < t.N)
				y[(long long)gcol * t.ldc + grow] = double(v[i]);
		}
	}
}

// pass 1, a warp's 32 full rows (tile rows row0 .. row0+31, all inside the
// matrix): the thread of tile row row0 + lane writes its 128-byte BX row of
// chunk (n0 + c0) / 32 into the warp's staging tile (hi at stg, lo at
// stg + 4096; 16-byte piece q of row r at r*128 + (q ^ (r % 8))*16, the
// TMA unit's 128-byte swizzle of a 1024-aligned box), and lane 0 stores
// both tiles.  Columns past N are the K padding of pass 2: zeros.
template <int BN>
__device__ __forceinline__ void store_chunk_tma(const TcArgs& a, const GemmTile& t, int row0, int c0,
                                                const float (&v)[32], unsigned stg, int lane)
{
	const int col0 = t.n0 + c0;
	if (col0 >= t.N)
		return;
	if (lane == 0)
		bulk_wait_read(); // the previous chunk's stores have read the tile
	__syncwarp();
	const unsigned rowaddr = stg + unsigned(lane) * 128u;
#pragma unroll
	for (int q = 0; q < 8; ++q) {
		float hv[4], lv[4];
#pragma unroll
		for (int e = 0; e < 4; ++e) {
			const float x = (col0 + 4 * q + e < t.N) ? v[4 * q + e] : 0.f;
			hv[e]         = tf32_rna(x);
			lv[e]         = tf32_rna(x - hv[e]);
		}
		const unsigned off = unsigned((q ^ (lane & 7)) << 4);
		st_shared_v4(rowaddr + off, hv[0], hv[1], hv[2], hv[3]);
		st_shared_v4(rowaddr + 4096u + off, lv[0], lv[1], lv[2], lv[3]);
	}
	fence_proxy_async();
	__syncwarp();
	if (lane == 0) {
		const int R = int(t.c_off >> 5) + (col0 >> 5) * t.ldc + t.m0 + row0;
		tma_store_2d(&a.C_hi_map, stg, R);
		tma_store_2d(&a.C_lo_map, stg + 4096u, R);
		bulk_commit();
	}
}

// the 4 epilogue warps only (named barrier 1)
__device__ __forceinline__ void epilogue_sync() { asm volatile("bar.sync 1, 128;\n" ::: "memory"); }

// AND of a flag over the 4 epilogue warps (named barrier 1), so that every
// epilogue thread takes the same branch after a bounded wait
__device__ __forceinline__ bool epilogue_all(bool v)
{
	unsigned out;
	asm volatile("{\n\t.reg .pred p, q;\n\t"
	             "setp.ne.u32 p, %1, 0;\n\t"
	             "bar.red.and.pred q, 1, 128, p;\n\t"
	             "selp.u32 %0, 1, 0, q;\n\t}\n"
	             : "=r"(out)
	             : "r"(unsigned(v))
	             : "memory");
	return out != 0;
}

// part of a K-split pass-2 tile: this thread's row of one 32-column chunk
// into the part's FP32 slot (row-major 128 x BN)
template <int BN>
__device__ __forceinline__ void store_partial(const TcArgs& a, const GemmTile& t, int row, int c0,
                                              const float (&v)[32])
{
	float* dst = a.partial + (size_t(t.slot + t.split_part) * 128 + size_t(row)) * BN + c0;
#pragma unroll
	for (int q = 0; q < 8; ++q)
		reinterpret_cast<float4*>(dst)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
}

// after every part of split tile t wrote its slot: sum the slots in part
// order (deterministic) and write y
template <int BN>
__device__ __forceinline__ void reduce_split(const TcArgs& a, const GemmTile& t, int row)
{
	const int grow = t.m0 + row;
	if (grow >= t.M)
		return;
	double* y = (a.io ? a.io->y : a.Cd) + t.c_off;
	for (int c0 = 0; c0 < BN && t.n0 + c0 < t.N; c0 += 32) {
		float s[32];
#pragma unroll
		for (int i = 0; i < 32; ++i)
			s[i] = 0.f;
		for (int p = 0; p < t.nsplit; ++p) {
			const float4* src = reinterpret_cast<const float4*>(
			    a.partial + (size_t(t.slot + p) * 128 + size_t(row)) * BN + c0);
#pragma unroll
			for (int q = 0; q < 8; ++q) {
				const float4 f = __ldcg(src + q);
				s[4 * q] += f.x;
				s[4 * q + 1] += f.y;
				s[4 * q + 2] += f.z;
				s[4 * q + 3] += f.w;
			}
		}
#pragma unroll
		for (int i = 0; i < 32; ++i) {
			const int gcol = t.n0 + c0 + i;
			if (gcol < t.N)
				y[(long long)gcol * t.ldc + grow] = double(s[i]);
		}
	}
}

template <int BN, bool PASS1>
__device__ void epilogue(const TcArgs& a, unsigned tmem, unsigned accf0, unsigned acce0,
                         volatile int* abort, unsigned staging)
{
	__shared__ int s_last;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int quarter = warp & 3; // TMEM lanes this warp may read
	const int row     = quarter * 32 + lane;
	const unsigned stg = staging + unsigned(warp - 2) * 8192u; // pass 1: this warp's tile
	unsigned  tc      = 0;
	bool      ok      = true;
	for (int ti = a.starts[blockIdx.x]; ti < a.starts[blockIdx.x + 1]; ++ti) {
		if (skip_tile(a, ti))
			continue;
		const GemmTile t     = a.tiles[ti];
		const int      total = tile_chunks(a, t);
		const int      grow  = t.m0 + row;
		float          v[32];
		if (total == 0) { // output tile without terms: zeros
#pragma unroll
			for (int i = 0; i < 32; ++i)
				v[i] = 0.f;
			for (int c0 = 0; c0 < BN; c0 += 32)
				store_chunk<BN, PASS1>(a, t, grow, c0, v);
			continue;
		}
		const unsigned b = tc & 1;
		// uniform over the epilogue warps: a wait that gave up in any of them
		// stops all (the split reduction below has unbounded named barriers)
		if (!epilogue_all(mbar_wait(accf0 + 8 * b, (tc >> 1) & 1, abort))) {
			ok = false;
			break;
		}
		tc_fence_after();
		const bool split = !PASS1 && t.nsplit >= 2;
		// pass 1: this warp's 32 rows all inside the matrix (the same for
		// every lane) -> staged TMA stores; a partial row group stores directly
		const bool staged = PASS1 && t.m0 + quarter * 32 + 32 <= t.M;
		for (int c0 = 0; c0 < BN; c0 += 32) {
			tmem_ld32(tmem + (unsigned(quarter * 32) << 16) + b * unsigned(BN) + unsigned(c0), v);
			if (split)
				store_partial<BN>(a, t, row, c0, v);
			else if (staged)
				store_chunk_tma<BN>(a, t, quarter * 32, c0, v, stg, lane);
			else
				store_chunk<BN, PASS1>(a, t, grow, c0, v);
		}
		tc_fence_before();
		__syncwarp();
		if (lane == 0)
			mbar_arrive(acce0 + 8 * b);
		++tc;
		if (split) {
			// the last part to finish sums every part's slot in order
			__threadfence();
			epilogue_sync();
			if (threadIdx.x == 64) {
				const unsigned old = atomicAdd(&a.arrive[t.split_tile], 1u);
				s_last             = old == unsigned(t.nsplit - 1);
				if (s_last)
					__threadfence();
			}
			epilogue_sync();
			if (s_last) {
				reduce_split<BN>(a, t, row);
				epilogue_sync();
				if (threadIdx.x == 64)
					a.arrive[t.split_tile] = 0u; // ready for the next launch
			}
		}
	}
	if (PASS1 && lane == 0)
		bulk_wait_all(); // this warp's TMA stores are written before the CTA exits
	if (!ok && lane == 0)
		give_up(abort, a.error);
}

template <int BN, int STAGES, bool PASS1>
__global__ void __launch_bounds__(kTcThreads, 1) tc_gemm_tf32x3_kernel(const __grid_constant__ TcArgs a)
{
	extern __shared__ unsigned char smem_raw[];
	__shared__ __align__(8) unsigned long long bars[2 * STAGES + 5];
	__shared__ unsigned                        tmem_slot;
	__shared__ volatile int                    abort_flag;

	const unsigned base   = (smem_addr(smem_raw) + 1023u) & ~1023u; // 1024-aligned stages
	const unsigned full0  = smem_addr(&bars[0]);
	const unsigned empty0 = smem_addr(&bars[STAGES]);
	const unsigned accf0  = smem_addr(&bars[2 * STAGES]);
	const unsigned acce0  = smem_addr(&bars[2 * STAGES + 2]);
	const unsigned drain  = smem_addr(&bars[2 * STAGES + 4]);
	const int      warp   = threadIdx.x >> 5;

	if (warp == 1) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
		                 smem_addr(&tmem_slot)),
		             "r"(unsigned(2 * BN))
		             : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
	}
	if (threadIdx.x == 0) {
		abort_flag = 0;
		for (int s = 0; s < STAGES; ++s) {
			mbar_init(full0 + 8 * s, 1);
			mbar_init(empty0 + 8 * s, 1);
		}
		for (int b = 0; b < 2; ++b) {
			mbar_init(accf0 + 8 * b, 1);
			mbar_init(acce0 + 8 * b, 4); // one arrival per epilogue warp
		}
		mbar_init(drain, 1);
		asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const unsigned tmem = tmem_slot;

	if (warp == 0) {
		if ((threadIdx.x & 31) == 0)
			producer<BN, STAGES>(a, base, full0, empty0, &abort_flag);
	} else if (warp == 1) {
		if ((threadIdx.x & 31) == 0)
			mma_issuer<BN, STAGES>(a, base, tmem, full0, empty0, accf0, acce0, drain, &abort_flag);
	} else {
		epilogue<BN, PASS1>(a, tmem, accf0, acce0, &abort_flag,
		                    base + unsigned(STAGES * TcLayout<BN>::STAGE_BYTES));
	}
	__syncwarp();
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	if (warp == 1)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
		             "r"(unsigned(2 * BN))
		             : "memory");
}

// x (FP64, patch order) -> TF32 hi/lo parts in the chunked layout
__global__ void __launch_bounds__(256)
split_x_kernel(const double* __restrict__ xin, const int* __restrict__ map, float* __restrict__ hi,
               float* __restrict__ lo, long long n, const StepIO* io)
{
	const double* x = io ? io->x : xin;
	for (long long e = blockIdx.x * 256LL + threadIdx.x; e < n; e += 256LL * gridDim.x) {
		const double v = x[e];
		const float  h = tf32_rna(float(v));
		const int    d = map[e];
		hi[d]          = h;
		lo[d]          = tf32_rna(float(v - double(h)));
	}
}

// FP64 packed operators -> chunked TF32 hi/lo layout (one block per job);
// the same rounding as the host's split_tf32
__global__ void __launch_bounds__(256)
pack_tf32_kernel(const double* __restrict__ ops, float* __restrict__ hi, float* __restrict__ lo,
                 const PackJob* __restrict__ jobs)
{
	const PackJob   j = jobs[blockIdx.x];
	const long long n = (long long)j.rows * j.cols;
	for (long long e = threadIdx.x; e < n; e += 256) {
		const int       q   = int(e % j.rows);
		const int       c   = int(e / j.rows);
		const double    v   = ops[j.src + q + (long long)c * j.ld];
		const long long row = j.swap ? c : j.row0 + q;
		const long long k   = j.swap ? q : c;
		const long long d   = j.dst + (k >> 5) * (long long)j.dst_rows * 32 + row * 32 + (k & 31);
		const float h = tf32_rna(float(v));
		hi[d]         = h;
		lo[d]         = tf32_rna(float(v - double(h)));
	}
}

// the ring, the 1 KB alignment slack and, in pass 1, four 8 KB staging
// tiles of the epilogue warps (1024-aligned: the ring's stages are)
template <int BN, int STAGES, bool PASS1> constexpr size_t tc_smem()
{
	return size_t(STAGES) * TcLayout<BN>::STAGE_BYTES + 1024 + (PASS1 ? 4 * 8192 : 0);
}

template <int BN, int STAGES, bool PASS1> cudaError_t tc_init_one()
{
	static_assert(tc_smem<BN, STAGES, PASS1>() + 256 <= 232448, "shared memory per CTA");
	return cudaFuncSetAttribute(tc_gemm_tf32x3_kernel<BN, STAGES, PASS1>,
	                            cudaFuncAttributeMaxDynamicSharedMemorySize,
	                            int(tc_smem<BN, STAGES, PASS1>()));
}

// ring depth: as many stages as fit in 227 KB with the 1 KB alignment slack
constexpr int kStages64  = 4; // 4 x 48 KB
constexpr int kStages128 = 3; // 3 x 64 KB

template <int BN, int STAGES, bool PASS1> void launch_one(const TcArgs& a, cudaStream_t stream)
{
	tc_gemm_tf32x3_kernel<BN, STAGES, PASS1><<<a.grid, kTcThreads, tc_smem<BN, STAGES, PASS1>(), stream>>>(a);
}

} // namespace

cudaError_t tc_init()
{
	cudaError_t e = tc_init_one<64, kStages64, true>();
	if (e == cudaSuccess)
		e = tc_init_one<64, kStages64, false>();
	if (e == cudaSuccess)
		e = tc_init_one<128, kStages128, true>();
	if (e == cudaSuccess)
		e = tc_init_one<128, kStages128, false>();
	return e;
}

cudaError_t tc_launch(const TcArgs& a, int bn, bool pass1, cudaStream_t stream)
{
	if (a.ntiles <= 0)
		return cudaSuccess;
	if (a.grid <= 0)
		return cudaErrorInvalidValue;
	if (bn == 64) {
		if (pass1)
			launch_one<64, kStages64, true>(a, stream);
		else
			launch_one<64, kStages64, false>(a, stream);
	} else if (bn == 128) {
		if (pass1)
			launch_one<128, kStages128, true>(a, stream);
		else
			launch_one<128, kStages128, false>(a, stream);
	} else {
		return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

cudaError_t tc_pack_ops(const double* ops, float* hi, float* lo, const PackJob* jobs, int njobs,
                        cudaStream_t stream)
{
	if (njobs <= 0)
		return cudaSuccess;
	pack_tf32_kernel<<<njobs, 256, 0, stream>>>(ops, hi, lo, jobs);
	return cudaGetLastError();
}

cudaError_t tc_split_x(const double* x, const int* map, float* hi, float* lo, long long n,
                       cudaStream_t stream, const StepIO* io)
{
	if (n <= 0)
		return cudaSuccess;
	long long blocks = (n + 255) / 256;
	if (blocks > 148 * 8)
		blocks = 148 * 8;
	split_x_kernel<<<int(blocks), 256, 0, stream>>>(x, map, hi, lo, n, io);
	return cudaGetLastError();
}

} // namespace dmrgpp
