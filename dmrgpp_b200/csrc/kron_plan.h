// Host-side schedule of one superblock sector's H*x as two grouped GEMM
// passes over the contributing (i,j,k) triples.
//
// Pass 1, one GEMM per input patch j (all output rows stacked, like the
// reference CPU batched path, BatchedGemmCpu.h:168-246):
//     BX_j (M_j x l_j) = Bstack_j (M_j x r_j) * X_j (r_j x l_j)
// where Bstack_j stacks B_k(i,j) for every contributing (i,k), in (i,k)
// order, and M_j is the sum of those r_i.
// Pass 2, one GEMM per output patch i (the plugin's second vbatch,
// apply_Htarget_sparse_not_ready.cpp:330-449):
//     Y_i (r_i x l_i) = sum over (j,k) of BX_j[rows of (i,k)] * A_k(i,j)^T
// The transposed A blocks are packed once (AT = A^T, l_j x l_i) so both
// passes read their B operand K-contiguous.
#pragma once

#include <algorithm>
#include <atomic>
#include <thread>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <string>
#include <memory>
#include <utility>
#include <vector>

#include <sched.h>

namespace dmrgpp {

// Host threads of the library's parallel host phases: DMRGPP_HOST_THREADS
// when it is set (1 to 256), otherwise the CPUs this process may run on (its
// affinity mask, so taskset, MPI binding and container CPU sets are
// honoured), at most 32.  Read once per process.
inline int host_threads()
{
	static const int n = [] {
		if (const char* e = std::getenv("DMRGPP_HOST_THREADS")) {
			const int v = std::atoi(e);
			if (v >= 1)
				return std::min(v, 256);
		}
		int       c = 0;
		cpu_set_t set;
		CPU_ZERO(&set);
		if (sched_getaffinity(0, sizeof set, &set) == 0)
			c = CPU_COUNT(&set);
		if (c <= 0)
			c = int(std::thread::hardware_concurrency());
		return std::max(1, std::min(c, 32));
	}();
	return n;
}

// f(0..n-1) on host_threads() threads (dynamic assignment; every f(i)
// writes its own disjoint output, so the result does not depend on the
// thread count)
template <class F> void parallel_for(size_t n, F f)
{
	size_t nt = size_t(host_threads());
	nt        = std::min(nt, n);
	if (nt < 2) {
		for (size_t i = 0; i < n; ++i)
			f(i);
		return;
	}
	std::atomic<size_t>      next { 0 };
	std::vector<std::thread> pool;
	for (size_t t = 0; t < nt; ++t)
		pool.emplace_back([&] {
			for (;;) {
				const size_t i = next.fetch_add(1);
				if (i >= n)
					break;
				f(i);
			}
		});
	for (std::thread& th : pool)
		th.join();
}

// One K-segment of an output tile: C += A(M x K) * B(K x N), column-major,
// offsets relative to the pass's A and B base pointers.
struct alignas(16) GemmSeg {
	long long a_off;
	long long b_off;
	int       lda;
	int       ldb;
	int       K;
	int       dep; // input patch j whose pass-1 result the segment reads (pass 2)
};

// One CTA's output tile [m0, m0+BM) x [n0, n0+BN) of an M x N matrix at
// c_off (leading dimension ldc), summed over segments [seg_begin, seg_end).
struct alignas(16) GemmTile {
	long long c_off;
	int       ldc;
	int       M;
	int       N;
	int       m0;
	int       n0;
	int       seg_begin;
	int       seg_end;
	// tensor-core pass 2 only: nsplit >= 2 marks part split_part of output
	// tile split_tile, cut along K at segment boundaries; its FP32 partial
	// goes to slot + split_part, the last part to arrive sums the slots
	int       nsplit;
	int       split_part;
	int       split_tile;
	int       slot;
};

// One work item of the persistent launch (kron_persistent.cu).
//   kind 0: pass-1 tile of input patch `producer` (segments index seg1)
//   kind 1: pass-2 output tile, whole K range (segments index pseg2)
//   kind 2: part `part` of `nsplit` K-slices of pass-2 output tile `tile`;
//           partial result goes to slot `slot + part`, the last part to
//           arrive sums the slots in order 0..nsplit-1 and writes the tile
struct alignas(16) KronItem {
	GemmSeg   seg0; // copy of the first segment (most items have only one)
	long long c_off;
	int       ldc;
	int       M;
	int       N;
	int       m0;
	int       n0;
	int       seg_begin;
	int       seg_end;
	int       kind;
	int       producer;
	int       tile;
	int       nsplit;
	int       slot;
	int       part;
	int       pad;
};

// Fused form (kron_fused.cu): one unit = one contributing triple (i,j,k)
// restricted to input columns [c0, c0 + cw) of X_j:
//     T  (rows x cw)  = B_k(i,j)[rows, :] * X_j[:, c0 .. c0+cw)
//     Y_i[rows, cols] += T * A_k(i,j)[cols, c0 .. c0+cw)^T
// Offsets point at element (row 0 of the (i,k) group, column 0) of
// Bstack_j, at X_j[0, c0], and at A^T_k(i,j)[c0, 0].
struct alignas(16) FusedUnit {
	long long b_off;
	long long x_off;
	long long at_off;
	int       ldb; // M_j (leading dimension of Bstack_j)
	int       rj;  // contraction of the first product (rows of X_j)
	int       lj;  // leading dimension of A^T_k(i,j) (= l_j)
	int       cw;  // columns of the unit (<= the configuration's unit width)
};

// One CTA of the fused launch: part `part` of `nparts` of the output tile
// [m0, m0+BM) x [n0, n0+BN) of Y_i (M = r_i rows, N = l_i columns, at y_off),
// summing units [u_begin, u_end).  The parts of one tile sit in one cluster
// at ranks rank0 .. rank0 + nparts - 1; nparts = 0 marks an empty slot.
struct alignas(16) FusedItem {
	long long y_off;
	int       M;
	int       N;
	int       m0;
	int       n0;
	int       u_begin;
	int       u_end;
	int       part;
	int       nparts;
	int       rank0;
	int       sector;
};

struct Triple {
	int i, j, k;
};

// Input and output vector of an H*x whose operands are chosen on the device
// (graph-replayed solver steps): the kernels read x and y from here at start.
struct StepIO {
	const double* x;
	double*       y;
};

// Host blocks of one contributing triple: A_k(i,j) (l_i x l_j) and B_k(i,j)
// (r_i x r_j), column-major with leading dimensions ldA, ldB.  Only valid
// while the caller's tables are (during create).
struct BlockRef {
	const double* A;
	size_t        ldA;
	const double* B;
	size_t        ldB;
};

// Layout of the mixed-precision (tensor-core) form of a sector.  Every
// operand is a "chunked K-major" matrix: rows padded to a multiple of 8 (Rp),
// K padded to a multiple of 32 with zeros, stored chunk by chunk (32 K values
// = 128 bytes per row, Rp rows per chunk): element (row, k) at
// chunked_offset(Rp, row, k).  Each operand buffer (packed operators, x
// split, BX split; hi and lo parts separately) is one 2-D tensor of the
// Tensor Memory Accelerator, [row][32 values], so rows (row0 .. row0 + box)
// of chunk c of a matrix are buffer rows (off/32 + c Rp + row0 ..): one
// tiled TMA load, written into shared memory with the 128-byte swizzle
// tcgen05.mma reads.  Rows of a tile past its matrix come from the next
// data in the buffer (or zeros past the buffer's end) and only feed
// discarded outputs.  Offsets are floats, multiples of 256.
//   pass 1: A = Bstack_j (Mp_j rows: the (i,k) groups, each r_i rows padded
//               to 8, at group_row[t]), K = r_j
//           B = X_j split (Lp_j = round8(l_j) rows), K = r_j
//           C = BX_j split (Mp_j rows, K = l_j for pass 2)
//   pass 2: A = the (i,k) group of BX_j, K = l_j
//           B = A_k(i,j)^T (round8(l_i) rows), K = l_j
//           C = Y_i, FP64 column-major
// GemmSeg of the mixed passes: a_off/b_off = buffer row of the matrix's
// chunk 0, row of the tile's row 0; lda/ldb = Rp (rows from one chunk to the
// next); K = K padded to 32.  GemmTile: ldc = padded rows of BX_j (pass 1)
// or r_i (pass 2).
inline long long round8(long long x) { return (x + 7) / 8 * 8; }
inline long long chunked_offset(long long rows_pad, long long row, long long k)
{
	return (k >> 5) * rows_pad * 32 + row * 32 + (k & 31);
}

struct MixedPlan {
	std::vector<long long> Mp;          // per input patch: padded rows of Bstack_j / BX_j
	std::vector<long long> group_row;   // per triple: first row of (i,k) in Bstack_j / BX_j
	std::vector<long long> bs_off;      // per input patch: Bstack_j in ops
	std::vector<long long> at_off;      // per triple: A^T in ops
	std::vector<long long> xs_off;      // per patch: X_j in the x split buffer
	std::vector<long long> bxs_off;     // per input patch: BX_j in the BX split buffer
	long long              ops_elems = 0, xs_elems = 0, bxs_elems = 0;
	std::vector<GemmSeg>   seg1, seg2;
	std::vector<GemmTile>  tile1, tile2;
	int                    bm = 128, bn = 64;
	int                    n_split_tiles = 0; // pass-2 output tiles cut along K
	long long              split_slots   = 0; // partial tiles of their parts
};

struct KronPlan {
	size_t np = 0, nop = 0;
	std::vector<long long> l, r;        // patch sizes
	std::vector<long long> xy_start;    // np+1 offsets into X / Y
	std::vector<Triple>    triples;     // contributing (i,j,k), (i,j,k) order
	std::vector<BlockRef>  blocks;      // per triple: host blocks (create time only)
	double                 f_alg = 0.0; // sum 2 r_i l_j (r_j + l_i)

	// packed operator buffer (doubles)
	std::vector<long long> bstack_off; // per input patch j
	std::vector<long long> M;          // rows of Bstack_j / BX_j
	std::vector<long long> at_off;     // per triple: packed A^T block
	long long              op_elems = 0;

	// intermediate BX buffer (doubles)
	std::vector<long long> bx_off;     // per input patch j
	std::vector<long long> row_off;    // per triple: first row of (i,k) in BX_j
	long long              bx_elems = 0;

	// launch lists of the two-launch form (pass 1 then pass 2)
	std::vector<GemmSeg>  seg1, seg2;
	std::vector<GemmTile> tile1, tile2;
	int                   bm = 64, bn = 64;

	// persistent form: pass-1 items first, then pass-2 items (K-split)
	std::vector<KronItem> items;
	std::vector<GemmSeg>  pseg2;         // pass-2 segments sliced per item
	std::vector<int>      n1_of_j;       // pass-1 items per input patch
	int                   n1_items = 0;
	int                   n_split_tiles = 0;
	long long             partial_slots = 0;

	MixedPlan mixed;

	// fused form: items cluster by cluster, and their units
	std::vector<FusedItem> fitems;
	std::vector<FusedUnit> funits;
	double                 f_max_part = 0.0; // modelled flops of the largest part

	long long dim() const { return xy_start.empty() ? 0 : xy_start.back(); }
};

// std::vector allocator that leaves elements uninitialised on resize (the
// packed operator buffer is fully written where it is read; skipping the
// zero fill of hundreds of MB halves the host side of create).
template <class T> struct NoInitAllocator : std::allocator<T> {
	template <class U> struct rebind {
		using other = NoInitAllocator<U>;
	};
	NoInitAllocator() = default;
	template <class U> NoInitAllocator(const NoInitAllocator<U>&) noexcept {}
	template <class U> void construct(U* p) noexcept { ::new (static_cast<void*>(p)) U; }
	template <class U, class... Args> void construct(U* p, Args&&... args)
	{
		::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
	}
};
using PackBuffer = std::vector<double, NoInitAllocator<double>>;

// Validates the plugin tables and builds the plan.  Returns an empty string on
// success, otherwise the reason.  pack_host (optional) receives the packed
// operator buffer (op_elems doubles).
std::string build_kron_plan(size_t               noperator,
                            size_t               npatches,
                            const size_t*        lsz,
                            const size_t*        rsz,
                            const double* const* A,
                            const size_t*        ldA,
                            const double* const* B,
                            const size_t*        ldB,
                            int                  bm,
                            int                  bn,
                            KronPlan&            plan,
                            PackBuffer*          pack_host);

// Appends the contributing triples of one plugin table (np patches, patch
// indices shifted by patch_offset) to triples/blocks, in (i,j,k) order:
// both blocks present and each with a nonzero entry (setup_nC.cpp:43-121).
// f_alg accumulates sum 2 r_i l_j (r_j + l_i).  Returns an error or "".
std::string collect_triples(size_t noperator, size_t np, const size_t* lsz, const size_t* rsz,
                            const double* const* A, const size_t* ldA, const double* const* B,
                            const size_t* ldB, int patch_offset, std::vector<Triple>& triples,
                            std::vector<BlockRef>& blocks, double& f_alg);

// Builds the plan from patch sizes and a triple list in (i,j,k) order (the
// union of independent sectors is such a list with shifted patch indices).
std::string build_kron_plan_triples(size_t noperator, size_t npatches, const size_t* lsz,
                                    const size_t* rsz, std::vector<Triple> triples,
                                    std::vector<BlockRef> blocks, double f_alg, int bm, int bn,
                                    KronPlan& plan, PackBuffer* pack_host);

// Builds plan.mixed for bn-wide tensor-core tiles from plan.blocks.  When
// ops_hi/ops_lo are given, packs the operators (hi and lo TF32 parts stored
// as floats); x_map (optional, dim entries) receives, for each element of the
// sector vector, its offset in the x split buffer.  Pass-2 tiles much longer
// than an even share of the work over `sms` SMs are cut along K at segment
// boundaries (small sectors would otherwise leave most SMs idle).
std::string build_mixed_plan(KronPlan& plan, int bn, std::vector<float>* ops_hi,
                             std::vector<float>* ops_lo, std::vector<int>* x_map,
                             int sms = 148);

// One block of the FP64 packed operators (column-major, leading dimension
// ld, rows x cols at src) into the chunked TF32 hi/lo layout: element (q, c)
// goes to row (swap ? c : row0 + q), K index (swap ? q : c) of the matrix
// at dst with dst_rows padded rows.
struct PackJob {
	long long src;
	long long dst;
	int       ld;
	int       rows;
	int       cols;
	int       dst_rows;
	int       row0;
	int       swap;
};

// The jobs that turn the FP64 packed operators of a planned sector (with
// plan.mixed built) into its chunked TF32 layout: per triple, its B block
// (rows of Bstack_j) and its A^T block.
std::vector<PackJob> mixed_pack_jobs(const KronPlan& plan);

// Staged upload of the FP64 packed operators at create time.  The caller's
// blocks are copied, column range by column range and contiguous
// (leading dimension = rows), into fixed-size chunks of pinned host memory;
// each chunk goes to the device in one copy, where a kernel moves every part
// to its place in the packed buffer (B blocks into Bstack_j, A blocks
// transposed into A^T).  One part = columns [col0, col0 + cols) of one block.
struct UploadJob {
	long long src;       // offset of the part in its chunk (doubles)
	long long dst;       // packed-buffer offset of element (0, col0) of the part
	int       rows;      // rows of the block
	int       cols;      // columns of the part
	int       ld_dst;    // leading dimension at dst
	int       transpose; // 0: (q, c) -> dst[q + c ld_dst]; 1: (q, c) -> dst[c + q ld_dst]
};

struct UploadPlan {
	long long              chunk_elems = 0; // capacity of one chunk (doubles)
	std::vector<UploadJob> jobs;            // in chunk order
	std::vector<size_t>    chunk_begin;     // jobs of chunk c: [chunk_begin[c], chunk_begin[c+1])
	std::vector<long long> chunk_fill;      // doubles used in chunk c
	std::vector<const double*> host_src;    // per job: the part's first column in the caller's block
	std::vector<long long> host_ld;         // per job: the caller's leading dimension
	size_t chunks() const { return chunk_fill.size(); }
};

// Cuts the blocks of plan.blocks into parts of at most max_job_elems doubles
// (at least one column) and fills chunks of chunk_elems doubles in triple
// order (B then A of each triple); a chunk is at least as large as the
// longest column.
UploadPlan build_upload_plan(const KronPlan& plan, long long chunk_elems, long long max_job_elems);

// Copies the parts of chunk c from the caller's blocks into buf (host side
// of the staged upload; jobs [first, last) of the chunk).
void fill_upload_chunk(const UploadPlan& up, size_t c, size_t first, size_t last, double* buf);

// Splits v into a TF32 high part and a TF32 remainder (host side of the
// operator packing; round to nearest, ties away from zero, like the
// device conversion cvt.rna.tf32.f32).
void split_tf32(double v, float* hi, float* lo);

// (Re)builds the two-launch tile lists seg1/tile1/seg2/tile2 of a planned
// sector for bm x bn output tiles.
void build_tile_lists(KronPlan& plan, int bm, int bn);

// Reorders the tiles of one tensor-core pass into per-CTA runs: CTA b of the
// persistent launch processes tiles [starts[b], starts[b+1]).  Tiles go,
// longest first, to the CTA with the least work so far (LPT; work of a tile =
// its k-chunks + 2 for the epilogue); within a run the longest tile comes
// first.  Returns the number of CTAs, min(bins, tiles.size()).
// Key of the autotuner's cache (autotune.cu): a hex FNV-1a hash of a coarse
// summary of the sector-size histogram (output-patch dimension at the work
// quartiles and maximum, by octave; the total work by half octave; the
// number of terms) and the GPU name.  Sectors of consecutive sweep steps,
// whose patch sizes change by a few states, mostly share a key.
std::string tuning_key(const KronPlan& P, const char* gpu);

int balance_tiles(std::vector<GemmTile>& tiles, const std::vector<GemmSeg>& segs, int bins,
                  std::vector<int>& starts);

// Most K-segments one work item may hold (they are staged in shared memory).
constexpr int kMaxItemSegs = 32;

// Builds plan.items / pseg2 / n1_of_j for a persistent launch of `grid`
// CTAs: pass-2 output tiles are cut into K-slices (multiples of bk, on any
// k boundary) when there are fewer than items_per_cta tiles per CTA.
void build_persistent_schedule(KronPlan& plan, int bk, int grid, int items_per_cta = 2);

// Checks the persistent work list against the buffers before a launch (the
// host-side bounds check of the debug mode, DMRGPP_VALIDATE=1): for every
// item, with tile x tile output tiles, the first and last element of each
// operand range (rows m0 .. min(m0 + tile, M) - 1, K, columns) lies inside
// its buffer (packed operators, x, BX, y), a pass-2 segment reads inside the
// BX of the patch it depends on, pass-1 items tile each BX_j exactly
// (n1_of_j of them), split parts agree on their tile and use their own
// slots, and no item holds more than kMaxItemSegs segments.  Returns "" or
// the first violation.
std::string validate_persistent_schedule(const KronPlan& plan, int tile);

// The same check for the fused work list (bm x bn output tiles, clusters of
// `cluster` CTAs): every non-empty item sits at rank rank0 + part of its
// cluster with rank0 + nparts <= cluster, its units are in range, and the
// first and last element of each unit's B, x and A^T ranges and of the
// item's Y tile lie inside their buffers.  Returns "" or the first violation.
std::string validate_fused_schedule(const KronPlan& plan, int bm, int bn, int cluster);

// The same check for the TF32x3 form (plan.mixed): every operand buffer a
// whole number of 32-float rows; for every tile and segment the K chunks a
// multiple of 32 and the leading dimensions of 8, the tile's valid rows
// inside its matrix, the start row of every tiled load inside its buffer;
// pass-1 outputs on 32-float rows with their staged stores and element
// stores inside the BX buffer; pass-2 stores inside y; split parts with
// slots in range and every part of a split tile present.  Returns "" or the
// first violation.
std::string validate_mixed_plan(const KronPlan& plan);

// DMRGPP_VALIDATE set to a nonzero number (read once per process).
bool validation_requested();

// Builds plan.fitems / funits for the fused launch: output tiles of bm rows
// and bn columns (columns past bn repeat the first product per column tile),
// units cw input columns wide, each tile's units cut into at most `cluster`
// parts of about equal modelled work (the target is the total over
// rounds x ctas parts, ctas = the CTAs resident at once), tiles packed whole
// into clusters of `cluster` CTAs (best fit, largest first).  sector_of_patch
// (optional, np entries) gives each output patch's sector for group handles.
void build_fused_schedule(KronPlan& plan, int bm, int bn, int cw, int cluster, int rounds,
                          int ctas, const std::vector<int>* sector_of_patch = nullptr);

} // namespace dmrgpp
