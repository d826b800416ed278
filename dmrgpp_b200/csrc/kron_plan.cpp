// Host-side planning of the two grouped-GEMM passes (see kron_plan.h).
#include "kron_plan.h"

#include <algorithm>
#include <cstdio>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <numeric>
#include <thread>
#include <tuple>
#include <utility>

namespace dmrgpp {

namespace {

constexpr long long kAlign = 32; // doubles (256 bytes) between packed blocks

long long align_up(long long x) { return (x + kAlign - 1) / kAlign * kAlign; }

bool has_nonzero(const double* m, size_t ld, size_t rows, size_t cols)
{
	if (!m)
		return false;
	for (size_t c = 0; c < cols; ++c) {
		const double* col = m + c * ld;
		for (size_t r = 0; r < rows; ++r)
			if (col[r] != 0.0)
				return true;
	}
	return false;
}

void add_tiles(std::vector<GemmTile>& tiles,
               long long              c_off,
               long long              ldc,
               long long              M,
               long long              N,
               int                    seg_begin,
               int                    seg_end,
               int                    bm,
               int                    bn)
{
	for (long long n0 = 0; n0 < N; n0 += bn)
		for (long long m0 = 0; m0 < M; m0 += bm) {
			GemmTile t {};
			t.c_off     = c_off;
			t.ldc       = int(ldc);
			t.M         = int(M);
			t.N         = int(N);
			t.m0        = int(m0);
			t.n0        = int(n0);
			t.seg_begin = seg_begin;
			t.seg_end   = seg_end;
			tiles.push_back(t);
		}
}

// Longest tiles first: with one CTA per tile the tail of the launch is then
// made of short tiles (largest-processing-time-first ordering).
void order_tiles(std::vector<GemmTile>& tiles, const std::vector<GemmSeg>& segs)
{
	auto cost = [&](const GemmTile& t) {
		long long k = 0;
		for (int s = t.seg_begin; s < t.seg_end; ++s)
			k += segs[s].K;
		return k;
	};
	std::stable_sort(tiles.begin(), tiles.end(), [&](const GemmTile& a, const GemmTile& b) {
		return cost(a) > cost(b);
	});
}

} // namespace

void build_tile_lists(KronPlan& plan, int bm, int bn)
{
	const size_t np = plan.np;
	const size_t nt = plan.triples.size();
	plan.bm         = bm;
	plan.bn         = bn;
	plan.seg1.clear();
	plan.seg2.clear();
	plan.tile1.clear();
	plan.tile2.clear();
	// pass 1: one segment and a tile grid per input patch with work
	for (size_t j = 0; j < np; ++j) {
		if (plan.M[j] == 0)
			continue;
		GemmSeg s {};
		s.a_off = plan.bstack_off[j];
		s.lda   = int(plan.M[j]);
		s.b_off = plan.xy_start[j];
		s.ldb   = int(plan.r[j]);
		s.K     = int(plan.r[j]);
		s.dep   = int(j);
		const int sb = int(plan.seg1.size());
		plan.seg1.push_back(s);
		add_tiles(plan.tile1, plan.bx_off[j], plan.M[j], plan.M[j], plan.l[j], sb, sb + 1, bm, bn);
	}
	order_tiles(plan.tile1, plan.seg1);

	// pass 2: per output patch, the (j,k) segments in plugin order; a patch
	// without contributions still gets tiles so Y_i is overwritten with 0
	size_t t = 0;
	for (size_t i = 0; i < np; ++i) {
		const int sb = int(plan.seg2.size());
		for (; t < nt && plan.triples[t].i == int(i); ++t) {
			const Triple& tr = plan.triples[t];
			GemmSeg       s {};
			s.a_off = plan.bx_off[tr.j] + plan.row_off[t];
			s.lda   = int(plan.M[tr.j]);
			s.b_off = plan.at_off[t];
			s.ldb   = int(plan.l[tr.j]);
			s.K     = int(plan.l[tr.j]);
			s.dep   = tr.j;
			plan.seg2.push_back(s);
		}
		const int se = int(plan.seg2.size());
		add_tiles(plan.tile2, plan.xy_start[i], plan.r[i], plan.r[i], plan.l[i], sb, se, bm, bn);
	}
	order_tiles(plan.tile2, plan.seg2);
}

std::string collect_triples(size_t noperator, size_t np, const size_t* lsz, const size_t* rsz,
                            const double* const* A, const size_t* ldA, const double* const* B,
                            const size_t* ldB, int patch_offset, std::vector<Triple>& triples,
                            std::vector<BlockRef>& blocks, double& f_alg)
{
	const size_t np2 = np * np;
	// present entries in (i,j,k) order; leading dimensions checked in order
	std::vector<size_t> cand;
	for (size_t i = 0; i < np; ++i)
		for (size_t j = 0; j < np; ++j)
			for (size_t k = 0; k < noperator; ++k) {
				const size_t t = i + j * np + k * np2;
				if (!A[t] || !B[t])
					continue;
				if (ldA[t] < lsz[i] || ldB[t] < rsz[i])
					return "leading dimension smaller than the block's rows at table entry "
					    + std::to_string(t);
				cand.push_back(t);
			}
	// the all-zero test reads every block: on all host cores
	std::vector<char> keep(cand.size(), 0);
	parallel_for(cand.size(), [&](size_t q) {
		const size_t t = cand[q];
		const size_t i = t % np, j = (t / np) % np;
		keep[q]        = has_nonzero(A[t], ldA[t], lsz[i], lsz[j]) && has_nonzero(B[t], ldB[t], rsz[i], rsz[j]);
	});
	for (size_t q = 0; q < cand.size(); ++q) {
		if (!keep[q])
			continue;
		const size_t t = cand[q];
		const size_t i = t % np, j = (t / np) % np, k = t / np2;
		triples.push_back({ int(i) + patch_offset, int(j) + patch_offset, int(k) });
		blocks.push_back({ A[t], ldA[t], B[t], ldB[t] });
		f_alg += 2.0 * double(rsz[i]) * double(lsz[j]) * (double(rsz[j]) + double(lsz[i]));
	}
	return std::string();
}

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
                            PackBuffer*          pack_host)
{
	if (noperator == 0 || npatches == 0)
		return "noperator and npatches must be >= 1";
	if (!lsz || !rsz || !A || !ldA || !B || !ldB)
		return "null table or size array";
	for (size_t p = 0; p < npatches; ++p)
		if (lsz[p] < 1 || rsz[p] < 1) // the reference asserts 1 <= size (setup_sparse_batch.cpp:70-71)
			return "patch " + std::to_string(p) + " has an empty left or right group";
	std::vector<Triple>   triples;
	std::vector<BlockRef> blocks;
	double                f_alg = 0.0;
	std::string msg = collect_triples(noperator, npatches, lsz, rsz, A, ldA, B, ldB, 0, triples,
	                                  blocks, f_alg);
	if (!msg.empty())
		return msg;
	return build_kron_plan_triples(noperator, npatches, lsz, rsz, std::move(triples),
	                               std::move(blocks), f_alg, bm, bn, plan, pack_host);
}

std::string build_kron_plan_triples(size_t noperator, size_t npatches, const size_t* lsz,
                                    const size_t* rsz, std::vector<Triple> triples,
                                    std::vector<BlockRef> blocks, double f_alg, int bm, int bn,
                                    KronPlan& plan, PackBuffer* pack_host)
{
	if (noperator == 0 || npatches == 0)
		return "noperator and npatches must be >= 1";
	if (triples.size() != blocks.size())
		return "triples and blocks differ in length";
	const size_t np = npatches;
	plan            = KronPlan();
	plan.np         = np;
	plan.nop        = noperator;
	plan.bm         = bm;
	plan.bn         = bn;
	plan.l.resize(np);
	plan.r.resize(np);
	plan.xy_start.assign(np + 1, 0);
	for (size_t p = 0; p < np; ++p) {
		if (lsz[p] < 1 || rsz[p] < 1)
			return "patch " + std::to_string(p) + " has an empty left or right group";
		if (lsz[p] > INT_MAX / 64 || rsz[p] > INT_MAX / 64)
			return "patch " + std::to_string(p) + " is too large";
		plan.l[p]            = (long long)lsz[p];
		plan.r[p]            = (long long)rsz[p];
		plan.xy_start[p + 1] = plan.xy_start[p] + plan.l[p] * plan.r[p];
	}
	for (size_t t = 0; t < triples.size(); ++t) {
		const Triple& tr = triples[t];
		if (tr.i < 0 || tr.j < 0 || size_t(tr.i) >= np || size_t(tr.j) >= np || tr.k < 0
		    || size_t(tr.k) >= noperator)
			return "triple " + std::to_string(t) + " out of range";
		if (t > 0) {
			const Triple& q = triples[t - 1];
			if (std::make_tuple(q.i, q.j, q.k) >= std::make_tuple(tr.i, tr.j, tr.k))
				return "triples not in (i,j,k) order";
		}
	}
	plan.triples = std::move(triples);
	plan.blocks  = std::move(blocks);
	plan.f_alg   = f_alg;

	const size_t nt = plan.triples.size();
	// pass-1 row layout: for each input patch j the rows of (i,k) stacked in
	// (i,k) order
	plan.M.assign(np, 0);
	plan.row_off.assign(nt, 0);
	for (size_t t = 0; t < nt; ++t) {
		const Triple& tr = plan.triples[t];
		plan.row_off[t]  = plan.M[tr.j];
		plan.M[tr.j] += plan.r[tr.i];
	}
	if (*std::max_element(plan.M.begin(), plan.M.end()) > INT_MAX / 2)
		return "stacked pass-1 operator too tall";

	// packed operators: Bstack_j then A^T blocks
	long long off = 0;
	plan.bstack_off.assign(np, 0);
	for (size_t j = 0; j < np; ++j) {
		plan.bstack_off[j] = off;
		off += align_up(plan.M[j] * plan.r[j]);
	}
	plan.at_off.assign(nt, 0);
	for (size_t t = 0; t < nt; ++t) {
		const Triple& tr = plan.triples[t];
		plan.at_off[t]   = off;
		off += align_up(plan.l[tr.j] * plan.l[tr.i]);
	}
	plan.op_elems = off;

	off = 0;
	plan.bx_off.assign(np, 0);
	for (size_t j = 0; j < np; ++j) {
		plan.bx_off[j] = off;
		off += align_up(plan.M[j] * plan.l[j]);
	}
	plan.bx_elems = off;

	if (pack_host) {
		pack_host->resize(size_t(plan.op_elems)); // every element that is read gets written
		double* P = pack_host->data();
		parallel_for(nt, [&](size_t t) {
			const Triple& tr = plan.triples[t];
			const BlockRef& bl = plan.blocks[t];
			// B_k(i,j) (r_i x r_j) into rows [row_off, row_off + r_i) of Bstack_j
			const long long Mj = plan.M[tr.j];
			double*         bs = P + plan.bstack_off[tr.j] + plan.row_off[t];
			const double*   b  = bl.B;
			for (long long c = 0; c < plan.r[tr.j]; ++c)
				for (long long q = 0; q < plan.r[tr.i]; ++q)
					bs[q + c * Mj] = b[q + c * (long long)bl.ldB];
			// A_k(i,j)^T (l_j x l_i), leading dimension l_j
			double*         at = P + plan.at_off[t];
			const double*   a  = bl.A;
			const long long lj = plan.l[tr.j];
			for (long long c = 0; c < plan.l[tr.i]; ++c)
				for (long long q = 0; q < lj; ++q)
					at[q + c * lj] = a[c + q * (long long)bl.ldA];
		});
	}

	build_tile_lists(plan, bm, bn);
	return std::string();
}

void build_persistent_schedule(KronPlan& plan, int bk, int grid, int items_per_cta)
{
	plan.items.clear();
	plan.pseg2.clear();
	plan.n1_of_j.assign(plan.np, 0);
	plan.n_split_tiles = 0;
	plan.partial_slots = 0;

	for (const GemmTile& t : plan.tile1) {
		KronItem w {};
		w.c_off     = t.c_off;
		w.ldc       = t.ldc;
		w.M         = t.M;
		w.N         = t.N;
		w.m0        = t.m0;
		w.n0        = t.n0;
		w.seg_begin = t.seg_begin;
		w.seg_end   = t.seg_end;
		w.kind      = 0;
		w.producer  = plan.seg1[t.seg_begin].dep;
		plan.n1_of_j[w.producer]++;
		plan.items.push_back(w);
	}
	plan.n1_items = int(plan.items.size());

	// K-slice length: none when the tiles alone give `items_per_cta` items per
	// CTA, otherwise aim at that many pass-2 items per CTA, at least 4 chunks
	// each; no item holds more than kMaxItemSegs segments
	long long total_k = 0;
	for (const GemmTile& t : plan.tile2)
		for (int s = t.seg_begin; s < t.seg_end; ++s)
			total_k += plan.seg2[s].K;
	long long k_target = 1LL << 40;
	const long long want = (long long)items_per_cta * grid;
	if ((long long)plan.tile2.size() < want && grid > 0) {
		k_target = total_k / want;
		k_target = std::max<long long>(k_target, 4LL * bk);
		k_target = (k_target + bk - 1) / bk * bk;
	}
	const int max_split = 16;

	std::vector<KronItem> p2;
	for (const GemmTile& t : plan.tile2) {
		long long kt = 0;
		for (int s = t.seg_begin; s < t.seg_end; ++s)
			kt += plan.seg2[s].K;
		int nsplit = int(std::min<long long>((kt + k_target - 1) / k_target, max_split));
		nsplit     = std::max(nsplit, 1);
		long long chunk = (kt + nsplit - 1) / nsplit;
		chunk           = std::max<long long>(bk, (chunk + bk - 1) / bk * bk);

		KronItem base {};
		base.c_off = t.c_off;
		base.ldc   = t.ldc;
		base.M     = t.M;
		base.N     = t.N;
		base.m0    = t.m0;
		base.n0    = t.n0;
		// cut the tile's segments into parts of `chunk` K (and <= kMaxItemSegs pieces)
		std::vector<KronItem> parts;
		int       s  = t.seg_begin;
		long long k0 = 0; // offset inside segment s
		do {
			KronItem w  = base;
			w.seg_begin = int(plan.pseg2.size());
			long long need = chunk;
			while (need > 0 && s < t.seg_end
			       && int(plan.pseg2.size()) - w.seg_begin < kMaxItemSegs) {
				const GemmSeg&  g    = plan.seg2[s];
				const long long take = std::min<long long>(need, g.K - k0);
				GemmSeg         piece = g;
				piece.a_off += k0 * g.lda; // A = BX_j columns k0..
				piece.b_off += k0;         // B = A^T rows k0.. (K-contiguous)
				piece.K = int(take);
				plan.pseg2.push_back(piece);
				need -= take;
				k0 += take;
				if (k0 == g.K) {
					++s;
					k0 = 0;
				}
			}
			w.seg_end = int(plan.pseg2.size());
			parts.push_back(w);
		} while (s < t.seg_end);
		if (parts.size() == 1) {
			parts[0].kind = 1;
			p2.push_back(parts[0]);
			continue;
		}
		const int tile_id = plan.n_split_tiles++;
		for (size_t q = 0; q < parts.size(); ++q) {
			parts[q].kind   = 2;
			parts[q].tile   = tile_id;
			parts[q].nsplit = int(parts.size());
			parts[q].slot   = int(plan.partial_slots);
			parts[q].part   = int(q);
			p2.push_back(parts[q]);
		}
		plan.partial_slots += (long long)parts.size();
	}
	auto cost = [&](const KronItem& w) {
		long long k = 0;
		for (int s = w.seg_begin; s < w.seg_end; ++s)
			k += plan.pseg2[s].K;
		return k;
	};
	std::stable_sort(p2.begin(), p2.end(),
	                 [&](const KronItem& a, const KronItem& b) { return cost(a) > cost(b); });
	plan.items.insert(plan.items.end(), p2.begin(), p2.end());
	for (KronItem& w : plan.items) {
		const std::vector<GemmSeg>& segs = w.kind == 0 ? plan.seg1 : plan.pseg2;
		if (w.seg_end > w.seg_begin)
			w.seg0 = segs[size_t(w.seg_begin)];
	}
}

bool validation_requested()
{
	static const bool on = [] {
		const char* e = std::getenv("DMRGPP_VALIDATE");
		return e && std::atoi(e) != 0;
	}();
	return on;
}

std::string validate_persistent_schedule(const KronPlan& plan, int tile)
{
	const long long dim = plan.dim(), ops = plan.op_elems, bx = plan.bx_elems;
	auto            at  = [](const char* what, size_t q) { return std::string(what) + " (item " + std::to_string(q) + ")"; };
	// [lo, hi] of rows [m0, m1) x k [0, K) of a column-major operand at off
	auto range_ok = [](long long off, long long r0, long long r1, long long cols, long long ld, long long lo,
	                   long long hi) {
		if (r1 <= r0 || cols <= 0)
			return true;
		const long long first = off + r0, last = off + (r1 - 1) + (cols - 1) * ld;
		return first >= lo && last < hi && ld >= 1;
	};
	if (plan.n1_items < 0 || size_t(plan.n1_items) > plan.items.size() || plan.n1_of_j.size() != plan.np)
		return "item counts";
	std::vector<long long> area(plan.np, 0);
	std::vector<int>       n1(plan.np, 0);
	std::vector<int>       slot_use(size_t(std::max<long long>(plan.partial_slots, 0)), 0);
	for (size_t q = 0; q < plan.items.size(); ++q) {
		const KronItem& w    = plan.items[q];
		const bool      p1   = q < size_t(plan.n1_items);
		const auto&     segs = p1 ? plan.seg1 : plan.pseg2;
		if (p1 != (w.kind == 0) || w.seg_begin < 0 || w.seg_end < w.seg_begin || size_t(w.seg_end) > segs.size())
			return at("kind or segment range", q);
		if (w.seg_end - w.seg_begin > kMaxItemSegs)
			return at("too many segments", q);
		if (w.M < 0 || w.N < 0 || w.m0 < 0 || w.n0 < 0 || w.m0 >= std::max(w.M, 1) || w.n0 >= std::max(w.N, 1))
			return at("tile origin", q);
		const long long m1 = std::min<long long>(w.m0 + tile, w.M), n1c = std::min<long long>(w.n0 + tile, w.N);
		const long long ncols = n1c - w.n0;
		// the output tile
		const long long out_lo = p1 ? 0 : 0, out_hi = p1 ? bx : dim;
		if (ncols > 0 && m1 > w.m0
		    && !range_ok(w.c_off + (long long)w.n0 * w.ldc, w.m0, m1, ncols, w.ldc, out_lo, out_hi))
			return at(p1 ? "BX store out of range" : "y store out of range", q);
		for (int e = w.seg_begin; e < w.seg_end; ++e) {
			const GemmSeg& g = segs[size_t(e)];
			if (g.dep < 0 || size_t(g.dep) >= plan.np || g.K < 0)
				return at("segment dependency", q);
			if (p1) {
				// A: Bstack_j rows m, k < K in the operators; B: X_j k < K, columns n
				if (!range_ok(g.a_off, w.m0, m1, g.K, g.lda, 0, ops))
					return at("pass-1 A load out of the operators", q);
				const long long xlo = plan.xy_start[size_t(g.dep)], xhi = plan.xy_start[size_t(g.dep) + 1];
				if (g.K > 0 && ncols > 0 && !range_ok(g.b_off + (long long)w.n0 * g.ldb, 0, g.K, ncols, g.ldb, xlo, xhi))
					return at("pass-1 x load out of X_j", q);
			} else {
				const long long blo = plan.bx_off[size_t(g.dep)];
				const long long bhi = blo + plan.M[size_t(g.dep)] * plan.l[size_t(g.dep)];
				if (!range_ok(g.a_off, w.m0, m1, g.K, g.lda, blo, bhi))
					return at("pass-2 BX load outside its dependency", q);
				if (g.K > 0 && ncols > 0 && !range_ok(g.b_off + (long long)w.n0 * g.ldb, 0, g.K, ncols, g.ldb, 0, ops))
					return at("pass-2 A^T load out of the operators", q);
			}
		}
		if (p1) {
			if (w.producer < 0 || size_t(w.producer) >= plan.np || w.seg_end - w.seg_begin != 1
			    || plan.seg1[size_t(w.seg_begin)].dep != w.producer)
				return at("pass-1 producer", q);
			const size_t j = size_t(w.producer);
			if (w.c_off != plan.bx_off[j] || w.M != plan.M[j] || w.N != plan.l[j] || w.ldc != plan.M[j])
				return at("pass-1 output is not BX_j", q);
			area[j] += (m1 - w.m0) * ncols;
			++n1[j];
		} else if (w.kind == 2) {
			if (w.nsplit < 2 || w.part < 0 || w.part >= w.nsplit || w.slot < 0
			    || (long long)w.slot + w.nsplit > plan.partial_slots || w.tile < 0 || w.tile >= plan.n_split_tiles)
				return at("split part", q);
			if (slot_use[size_t(w.slot + w.part)]++)
				return at("split slot used twice", q);
		} else if (w.kind != 1) {
			return at("item kind", q);
		}
	}
	for (size_t j = 0; j < plan.np; ++j)
		if (n1[j] != plan.n1_of_j[j] || area[j] != plan.M[j] * plan.l[j])
			return "pass-1 tiles do not cover BX_" + std::to_string(j) + " exactly once";
	for (size_t s = 0; s < slot_use.size(); ++s)
		if (slot_use[s] != 1)
			return "split slot " + std::to_string(s) + " unused";
	return "";
}

std::string validate_fused_schedule(const KronPlan& plan, int bm, int bn, int cluster)
{
	const long long dim = plan.dim(), ops = plan.op_elems;
	const auto&     I   = plan.fitems;
	const auto&     U   = plan.funits;
	auto at = [](const char* what, size_t q) { return std::string(what) + " (item " + std::to_string(q) + ")"; };
	auto in = [](long long first, long long last, long long hi) { return first >= 0 && last >= first && last < hi; };
	if (cluster < 1 || I.size() % size_t(cluster) != 0)
		return "items are not whole clusters";
	for (size_t q = 0; q < I.size(); ++q) {
		const FusedItem& it = I[q];
		if (it.nparts == 0)
			continue;
		const int rank = int(q % size_t(cluster));
		if (it.nparts < 0 || it.part < 0 || it.part >= it.nparts || it.rank0 < 0 || it.rank0 + it.nparts > cluster
		    || it.rank0 + it.part != rank)
			return at("part placement", q);
		if (it.u_begin < 0 || it.u_end < it.u_begin || size_t(it.u_end) > U.size())
			return at("unit range", q);
		if (it.M < 1 || it.N < 1 || it.m0 < 0 || it.n0 < 0 || it.m0 >= it.M || it.n0 >= it.N)
			return at("tile origin", q);
		const long long Mt = std::min<long long>(bm, it.M - it.m0), Nt = std::min<long long>(bn, it.N - it.n0);
		if (!in(it.y_off + (long long)it.n0 * it.M + it.m0, it.y_off + (long long)(it.n0 + Nt - 1) * it.M + it.m0 + Mt - 1,
		        dim))
			return at("y tile out of range", q);
		for (int u = it.u_begin; u < it.u_end; ++u) {
			const FusedUnit& d = U[size_t(u)];
			if (d.rj < 1 || d.cw < 1 || d.lj < d.cw || d.ldb < 1)
				return at("unit shape", q);
			if (!in(d.b_off + it.m0, d.b_off + (long long)(d.rj - 1) * d.ldb + it.m0 + Mt - 1, ops))
				return at("B load out of the operators", q);
			if (!in(d.x_off, d.x_off + (long long)(d.cw - 1) * d.rj + d.rj - 1, dim))
				return at("x load out of range", q);
			if (!in(d.at_off + (long long)it.n0 * d.lj, d.at_off + (long long)(it.n0 + Nt - 1) * d.lj + d.cw - 1, ops))
				return at("A^T load out of the operators", q);
		}
	}
	return "";
}

std::string validate_mixed_plan(const KronPlan& plan)
{
	const MixedPlan& mp = plan.mixed;
	const long long  D  = plan.dim();
	const int        BM = mp.bm, BN = mp.bn;
	if (mp.ops_elems % 32 || mp.xs_elems % 32 || mp.bxs_elems % 32)
		return "an operand buffer is not a whole number of 32-float rows";
	std::map<int, std::vector<int>> parts; // split tile -> its parts seen
	std::map<int, int>              nsplit;
	auto pass = [&](const std::vector<GemmSeg>& segs, const std::vector<GemmTile>& tiles, long long arows,
	                long long brows, bool pass1) -> std::string {
		const char* name = pass1 ? "pass 1" : "pass 2";
		for (size_t q = 0; q < tiles.size(); ++q) {
			const GemmTile& t   = tiles[q];
			auto            bad = [&](const char* what) {
                return std::string(name) + ": " + what + " (tile " + std::to_string(q) + ")";
			};
			if (t.seg_begin < 0 || t.seg_end < t.seg_begin || size_t(t.seg_end) > segs.size())
				return bad("segment range");
			if (t.M < 1 || t.N < 1 || t.m0 < 0 || t.n0 < 0 || t.m0 >= t.M || t.n0 >= t.N)
				return bad("tile origin");
			const int vm = std::min(BM, t.M - t.m0), vn = std::min(BN, t.N - t.n0);
			for (int e = t.seg_begin; e < t.seg_end; ++e) {
				const GemmSeg& g = segs[size_t(e)];
				if (g.K < 0 || g.K % 32 != 0 || g.lda <= 0 || g.ldb <= 0 || g.lda % 8 != 0 || g.ldb % 8 != 0)
					return bad("segment fields");
				if (t.m0 + vm > g.lda || t.n0 + vn > g.ldb)
					return bad("valid rows past the matrix");
				if (g.K == 0)
					continue;
				const long long c1 = g.K / 32 - 1;
				const long long ya0 = g.a_off + t.m0, ya1 = ya0 + c1 * g.lda;
				const long long yb0 = g.b_off + t.n0, yb1 = yb0 + c1 * g.ldb;
				if (ya0 < 0 || yb0 < 0 || ya1 >= arows || yb1 >= brows || ya1 > INT_MAX || yb1 > INT_MAX)
					return bad("a tiled load starts outside its buffer");
			}
			const long long last_c0 = t.n0 + 32LL * ((vn - 1) / 32); // first column of the last 32-column group
			if (pass1) {
				if (t.c_off < 0 || t.c_off % 32 != 0)
					return bad("BX matrix not on a 32-float row");
				int qmax = -1; // the last full 32-row group of the tile
				for (int g = 0; g < 4; ++g)
					if (t.m0 + 32 * g + 32 <= t.M && 32 * g < BM)
						qmax = g;
				if (qmax >= 0) {
					const long long R = t.c_off / 32 + (last_c0 >> 5) * t.ldc + t.m0 + 32 * qmax;
					if (R < 0 || R > INT_MAX || (R + 32) * 32 > mp.bxs_elems)
						return bad("staged BX store outside the buffer");
				}
				const long long o = t.c_off + (last_c0 >> 5) * (long long)t.ldc * 32 + (long long)(t.m0 + vm - 1) * 32 + 31;
				if (o >= mp.bxs_elems)
					return bad("BX store out of bounds");
			} else {
				const long long o0 = t.c_off + (long long)t.n0 * t.ldc + t.m0;
				const long long o1 = t.c_off + (long long)(t.n0 + vn - 1) * t.ldc + t.m0 + vm - 1;
				if (o0 < 0 || o1 >= D)
					return bad("y store out of bounds");
				if (t.nsplit >= 2) {
					if (t.slot < 0 || t.split_part < 0 || t.split_part >= t.nsplit
					    || (long long)t.slot + t.nsplit > mp.split_slots || t.split_tile < 0
					    || t.split_tile >= mp.n_split_tiles)
						return bad("split slot out of range");
					parts[t.split_tile].push_back(t.split_part);
					nsplit[t.split_tile] = t.nsplit;
				}
			}
		}
		return "";
	};
	std::string v = pass(mp.seg1, mp.tile1, mp.ops_elems / 32, mp.xs_elems / 32, true);
	if (v.empty())
		v = pass(mp.seg2, mp.tile2, mp.bxs_elems / 32, mp.ops_elems / 32, false);
	if (!v.empty())
		return v;
	if (int(parts.size()) != mp.n_split_tiles)
		return "split tiles without parts";
	for (auto& kv : parts) {
		std::sort(kv.second.begin(), kv.second.end());
		for (int p = 0; p < int(kv.second.size()); ++p)
			if (kv.second[size_t(p)] != p)
				return "split tile " + std::to_string(kv.first) + " with a missing or repeated part";
		if (int(kv.second.size()) != nsplit[kv.first])
			return "split tile " + std::to_string(kv.first) + " missing parts";
	}
	return "";
}

void build_fused_schedule(KronPlan& plan, int bm, int bn, int cw, int cluster, int rounds,
                          int ctas, const std::vector<int>* sector_of_patch)
{
	plan.fitems.clear();
	plan.funits.clear();
	plan.f_max_part = 0.0;
	const size_t np = plan.np, nt = plan.triples.size();
	// contributing triples of output patch i: [tri_begin[i], tri_begin[i+1])
	std::vector<size_t> tri_begin(np + 1, nt);
	for (size_t t = nt; t-- > 0;)
		tri_begin[size_t(plan.triples[t].i)] = t;
	for (size_t i = np; i-- > 0;)
		if (tri_begin[i] > tri_begin[i + 1])
			tri_begin[i] = tri_begin[i + 1];

	auto up = [](long long x, long long q) { return (x + q - 1) / q * q; };
	struct Tile {
		int       i, m0, n0;
		size_t    u_begin, u_end; // in plan.funits
		double    work;
		int       parts;
		std::vector<size_t> cut; // parts + 1 unit boundaries
	};
	std::vector<Tile>   tiles;
	std::vector<double> uwork; // per unit: modelled flops
	// modelled cost of one k-step (16 of the contraction) apart from its flops
	const double step_cost = 2.0 * 32 * 32 * 16;
	double total = 0.0;
	for (size_t i = 0; i < np; ++i) {
		const long long M = plan.r[i], N = plan.l[i];
		for (long long m0 = 0; m0 < M; m0 += bm)
			for (long long n0 = 0; n0 < N; n0 += bn) {
				Tile tl {};
				tl.i       = int(i);
				tl.m0      = int(m0);
				tl.n0      = int(n0);
				tl.u_begin = plan.funits.size();
				const double bme = double(up(std::min<long long>(bm, M - m0), 8));
				const double bne = double(up(std::min<long long>(bn, N - n0), 8));
				for (size_t t = tri_begin[i]; t < tri_begin[i + 1]; ++t) {
					const Triple&   tr = plan.triples[t];
					const long long rj = plan.r[tr.j], lj = plan.l[tr.j];
					for (long long c0 = 0; c0 < lj; c0 += cw) {
						FusedUnit u {};
						u.cw     = int(std::min<long long>(cw, lj - c0));
						u.b_off  = plan.bstack_off[tr.j] + plan.row_off[t];
						u.ldb    = int(plan.M[tr.j]);
						u.rj     = int(rj);
						u.x_off  = plan.xy_start[tr.j] + c0 * rj;
						u.at_off = plan.at_off[t] + c0;
						u.lj     = int(lj);
						plan.funits.push_back(u);
						const double k1 = double(up(rj, 16)), k2 = double(up(u.cw, 16));
						const double w  = 2.0 * bme * double(up(u.cw, 8)) * k1 + 2.0 * bme * bne * k2
						    + step_cost * (k1 + k2) / 16.0;
						uwork.push_back(w);
						tl.work += w;
					}
				}
				tl.u_end = plan.funits.size();
				total += tl.work;
				tiles.push_back(std::move(tl));
			}
	}
	const double target = total / double(std::max(1, rounds * ctas));
	for (Tile& tl : tiles) {
		const size_t nu = tl.u_end - tl.u_begin;
		int          p  = target > 0.0 ? int(std::ceil(tl.work / target - 1e-9)) : 1;
		p               = std::max(1, std::min<int>(p, cluster));
		p               = int(std::min<size_t>(size_t(p), std::max<size_t>(nu, 1)));
		tl.parts        = p;
		// cut where the running work crosses q / p of the tile's work (the
		// nearer unit boundary), keeping every part non-empty
		tl.cut.assign(size_t(p) + 1, tl.u_begin);
		tl.cut[size_t(p)] = tl.u_end;
		double acc  = 0.0;
		size_t u    = tl.u_begin;
		for (int q = 1; q < p; ++q) {
			const double goal = tl.work * q / p;
			while (u < tl.u_end - size_t(p - q) && acc + uwork[u] * 0.5 < goal) {
				acc += uwork[u];
				++u;
			}
			if (u <= tl.cut[size_t(q - 1)]) { // at least one unit per part
				acc += uwork[u];
				++u;
			}
			tl.cut[size_t(q)] = u;
		}
		for (int q = 0; q < p; ++q) {
			double w = 0.0;
			for (size_t v = tl.cut[size_t(q)]; v < tl.cut[size_t(q) + 1]; ++v)
				w += uwork[v];
			plan.f_max_part = std::max(plan.f_max_part, w);
		}
	}
	// whole tiles into clusters: largest part count first, best fit
	std::vector<size_t> order(tiles.size());
	for (size_t q = 0; q < order.size(); ++q)
		order[q] = q;
	std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
		if (tiles[a].parts != tiles[b].parts)
			return tiles[a].parts > tiles[b].parts;
		return tiles[a].work > tiles[b].work;
	});
	struct Cl {
		int                 used = 0;
		double              heaviest = 0.0;
		std::vector<size_t> tiles;
	};
	std::vector<Cl>                  cls;
	std::vector<std::vector<size_t>> by_free(size_t(cluster) + 1); // clusters by free slots
	for (size_t q : order) {
		const Tile& tl   = tiles[q];
		size_t      cidx = SIZE_MAX;
		for (int f = tl.parts; f < cluster && cidx == SIZE_MAX; ++f)
			if (!by_free[size_t(f)].empty()) {
				cidx = by_free[size_t(f)].back();
				by_free[size_t(f)].pop_back();
			}
		if (cidx == SIZE_MAX) {
			cidx = cls.size();
			cls.emplace_back();
		}
		Cl& c = cls[cidx];
		c.used += tl.parts;
		c.heaviest = std::max(c.heaviest, tl.work / tl.parts);
		c.tiles.push_back(q);
		const int free = cluster - c.used;
		if (free > 0)
			by_free[size_t(free)].push_back(cidx);
	}
	std::vector<size_t> corder(cls.size());
	for (size_t q = 0; q < corder.size(); ++q)
		corder[q] = q;
	std::stable_sort(corder.begin(), corder.end(),
	                 [&](size_t a, size_t b) { return cls[a].heaviest > cls[b].heaviest; });
	plan.fitems.reserve(cls.size() * size_t(cluster));
	for (size_t c : corder) {
		int rank = 0;
		for (size_t q : cls[c].tiles) {
			const Tile& tl = tiles[q];
			const int   i  = tl.i;
			for (int p = 0; p < tl.parts; ++p) {
				FusedItem it {};
				it.y_off   = plan.xy_start[size_t(i)];
				it.M       = int(plan.r[size_t(i)]);
				it.N       = int(plan.l[size_t(i)]);
				it.m0      = tl.m0;
				it.n0      = tl.n0;
				it.u_begin = int(tl.cut[size_t(p)]);
				it.u_end   = int(tl.cut[size_t(p) + 1]);
				it.part    = p;
				it.nparts  = tl.parts;
				it.rank0   = rank;
				it.sector  = sector_of_patch ? (*sector_of_patch)[size_t(i)] : 0;
				plan.fitems.push_back(it);
			}
			rank += tl.parts;
		}
		for (; rank < cluster; ++rank) {
			FusedItem it {};
			it.nparts = 0;
			plan.fitems.push_back(it);
		}
	}
}

} // namespace dmrgpp

namespace dmrgpp {

namespace {

float tf32_round(float f)
{
	unsigned u;
	std::memcpy(&u, &f, 4);
	if ((u & 0x7f800000u) != 0x7f800000u) // finite: round the magnitude half away from zero
		u = (u + 0x1000u) & ~0x1fffu;
	float r;
	std::memcpy(&r, &u, 4);
	return r;
}

long long round32(long long x) { return (x + 31) / 32 * 32; }

void add_tc_tiles(std::vector<GemmTile>& tiles, long long c_off, long long ldc, long long M,
                  long long N, int sb, int se, int bm, int bn)
{
	for (long long n0 = 0; n0 < N; n0 += bn)
		for (long long m0 = 0; m0 < M; m0 += bm) {
			GemmTile t {};
			t.c_off     = c_off;
			t.ldc       = int(ldc);
			t.M         = int(M);
			t.N         = int(N);
			t.m0        = int(m0);
			t.n0        = int(n0);
			t.seg_begin = sb;
			t.seg_end   = se;
			tiles.push_back(t);
		}
}

} // namespace

namespace {
int octave(double x) { return x >= 1.0 ? int(std::floor(std::log2(x))) : 0; }
} // namespace

// FNV-1a over a coarse summary of the sector's size histogram: the patch
// dimension (max(l_i, r_i) of the output patch) at the quartiles and the
// maximum of the work-weighted distribution, one bucket per octave; the
// total work in half-octave buckets; the number of terms; the GPU name.
// These set what the configurations trade off (tile padding against
// tiles per SM), and they move little between consecutive sweep steps,
// whose patch sizes change by a few states, so those sectors share an
// entry.
std::string tuning_key(const KronPlan& P, const char* gpu)
{
	std::vector<std::pair<long long, double>> w; // (patch dimension, work)
	double                                    total = 0.0;
	long long                                 dmax  = 0;
	for (const auto& t : P.triples) {
		const long long d = std::max(P.l[size_t(t.i)], P.r[size_t(t.i)]);
		const double    f = 2.0 * double(P.r[size_t(t.i)]) * double(P.l[size_t(t.j)])
		    * double(P.r[size_t(t.j)] + P.l[size_t(t.i)]);
		w.push_back({ d, f });
		total += f;
		dmax = std::max(dmax, d);
	}
	std::sort(w.begin(), w.end());
	long long q[3] = { 0, 0, 0 };
	double    acc  = 0.0;
	int       k    = 0;
	for (const auto& e : w) {
		acc += e.second;
		while (k < 3 && acc >= total * 0.25 * (k + 1))
			q[k++] = e.first;
	}
	unsigned long long h   = 1469598103934665603ull;
	auto               mix = [&](unsigned long long v) {
                for (int b = 0; b < 8; ++b) {
                        h ^= (v >> (8 * b)) & 0xffu;
                        h *= 1099511628211ull;
                }
	};
	mix(P.nop);
	for (long long v : q)
		mix((unsigned long long)octave(double(v)));
	mix((unsigned long long)octave(double(dmax)));
	mix((unsigned long long)(total > 1.0 ? int(std::floor(2.0 * std::log2(total))) : 0));
	for (const char* c = gpu; *c; ++c)
		mix((unsigned long long)(unsigned char)*c);
	char buf[32];
	std::snprintf(buf, sizeof(buf), "%016llx", h);
	return buf;
}

UploadPlan build_upload_plan(const KronPlan& plan, long long chunk_elems, long long max_job_elems)
{
	UploadPlan up;
	long long  longest = 1;
	for (const Triple& tr : plan.triples)
		longest = std::max({ longest, plan.r[tr.i], plan.l[tr.i] });
	up.chunk_elems = std::max(chunk_elems, longest);
	max_job_elems  = std::max<long long>(max_job_elems, 1);

	long long fill = 0; // doubles used in the open chunk
	up.chunk_begin.push_back(0);
	auto close_chunk = [&] {
		up.chunk_fill.push_back(fill);
		up.chunk_begin.push_back(up.jobs.size());
		fill = 0;
	};
	// the block rows x cols at src (leading dimension ld) in parts
	auto add_block = [&](const double* src, long long ld, long long rows, long long cols,
	                     long long dst, int ld_dst, int transpose) {
		const long long job_cols = std::max<long long>(1, max_job_elems / rows);
		for (long long c0 = 0; c0 < cols;) {
			long long room = (up.chunk_elems - fill) / rows;
			if (room < 1) {
				close_chunk();
				room = up.chunk_elems / rows;
			}
			const long long n = std::min({ cols - c0, job_cols, room });
			UploadJob       j;
			j.src       = fill;
			j.dst       = dst + (transpose ? c0 : c0 * ld_dst);
			j.rows      = int(rows);
			j.cols      = int(n);
			j.ld_dst    = ld_dst;
			j.transpose = transpose;
			up.jobs.push_back(j);
			up.host_src.push_back(src + c0 * ld);
			up.host_ld.push_back(ld);
			fill += rows * n;
			c0 += n;
		}
	};
	for (size_t t = 0; t < plan.triples.size(); ++t) {
		const Triple&   tr = plan.triples[t];
		const BlockRef& bl = plan.blocks[t];
		// B_k(i,j) (r_i x r_j) into rows [row_off, row_off + r_i) of Bstack_j
		add_block(bl.B, (long long)bl.ldB, plan.r[tr.i], plan.r[tr.j],
		          plan.bstack_off[tr.j] + plan.row_off[t], int(plan.M[tr.j]), 0);
		// A_k(i,j) (l_i x l_j) transposed into A^T (l_j x l_i, leading dimension l_j)
		add_block(bl.A, (long long)bl.ldA, plan.l[tr.i], plan.l[tr.j], plan.at_off[t],
		          int(plan.l[tr.j]), 1);
	}
	if (fill > 0 || up.chunk_fill.empty())
		close_chunk();
	return up;
}

void fill_upload_chunk(const UploadPlan& up, size_t c, size_t first, size_t last, double* buf)
{
	for (size_t q = up.chunk_begin[c] + first; q < up.chunk_begin[c] + last; ++q) {
		const UploadJob& j   = up.jobs[q];
		const double*    src = up.host_src[q];
		const long long  ld  = up.host_ld[q];
		double*          dst = buf + j.src;
		if (ld == j.rows) {
			std::memcpy(dst, src, size_t(j.rows) * size_t(j.cols) * sizeof(double));
		} else {
			for (int c2 = 0; c2 < j.cols; ++c2)
				std::memcpy(dst + (long long)c2 * j.rows, src + c2 * ld, size_t(j.rows) * sizeof(double));
		}
	}
}

void split_tf32(double v, float* hi, float* lo)
{
	const float h = tf32_round(float(v));
	*hi           = h;
	*lo           = tf32_round(float(v - double(h)));
}

std::string build_mixed_plan(KronPlan& plan, int bn, std::vector<float>* ops_hi,
                             std::vector<float>* ops_lo, std::vector<int>* x_map, int sms)
{
	MixedPlan& mp   = plan.mixed;
	mp              = MixedPlan();
	mp.bn           = bn;
	const size_t np = plan.np, nt = plan.triples.size();
	// (i,k) groups of Bstack_j / BX_j, in triple order, each padded to 8 rows
	mp.Mp.assign(np, 0);
	mp.group_row.assign(nt, 0);
	for (size_t t = 0; t < nt; ++t) {
		const Triple& tr = plan.triples[t];
		mp.group_row[t]  = mp.Mp[tr.j];
		mp.Mp[tr.j] += round8(plan.r[tr.i]);
	}
	long long off = 0;
	mp.bs_off.assign(np, 0);
	for (size_t j = 0; j < np; ++j) {
		mp.bs_off[j] = off;
		off += mp.Mp[j] * round32(plan.r[j]);
	}
	mp.at_off.assign(nt, 0);
	for (size_t t = 0; t < nt; ++t) {
		mp.at_off[t] = off;
		off += round8(plan.l[plan.triples[t].i]) * round32(plan.l[plan.triples[t].j]);
	}
	mp.ops_elems = off;
	off          = 0;
	mp.xs_off.assign(np, 0);
	for (size_t p = 0; p < np; ++p) {
		mp.xs_off[p] = off;
		off += round8(plan.l[p]) * round32(plan.r[p]);
	}
	mp.xs_elems = off;
	off         = 0;
	mp.bxs_off.assign(np, 0);
	for (size_t j = 0; j < np; ++j) {
		mp.bxs_off[j] = off;
		off += mp.Mp[j] * round32(plan.l[j]);
	}
	mp.bxs_elems = off;
	if (mp.ops_elems > INT_MAX || mp.xs_elems > INT_MAX || mp.bxs_elems > INT_MAX)
		return "sector too large for the mixed-precision layout";

	if (ops_hi && ops_lo) {
		ops_hi->assign(size_t(mp.ops_elems), 0.0f);
		ops_lo->assign(size_t(mp.ops_elems), 0.0f);
		float* H = ops_hi->data();
		float* L = ops_lo->data();
		for (size_t t = 0; t < nt; ++t) {
			const Triple&   tr = plan.triples[t];
			const BlockRef& bl = plan.blocks[t];
			// Bstack_j row (group_row + q), K index c: B_k(i,j)(q, c)
			const double*   b  = bl.B;
			const long long Mj = mp.Mp[tr.j];
			for (long long q = 0; q < plan.r[tr.i]; ++q) {
				const long long row = mp.group_row[t] + q;
				for (long long c = 0; c < plan.r[tr.j]; ++c) {
					const long long o = mp.bs_off[tr.j] + chunked_offset(Mj, row, c);
					split_tf32(b[q + c * (long long)bl.ldB], H + o, L + o);
				}
			}
			// A^T row n (< l_i), K index k (< l_j): A_k(i,j)(n, k)
			const double*   a  = bl.A;
			const long long Ri = round8(plan.l[tr.i]);
			for (long long n = 0; n < plan.l[tr.i]; ++n)
				for (long long k = 0; k < plan.l[tr.j]; ++k) {
					const long long o = mp.at_off[t] + chunked_offset(Ri, n, k);
					split_tf32(a[n + k * (long long)bl.ldA], H + o, L + o);
				}
		}
	}
	if (x_map) {
		// X_p(iR, iL) -> row iL, K index iR of the x split
		x_map->assign(size_t(plan.dim()), 0);
		for (size_t p = 0; p < np; ++p) {
			const long long Lp = round8(plan.l[p]);
			for (long long n = 0; n < plan.l[p]; ++n)
				for (long long k = 0; k < plan.r[p]; ++k)
					(*x_map)[size_t(plan.xy_start[p] + k + n * plan.r[p])]
					    = int(mp.xs_off[p] + chunked_offset(Lp, n, k));
		}
	}

	// pass 1: C = BX_j split (every padded row, K-chunks of l_j)
	for (size_t j = 0; j < np; ++j) {
		if (mp.Mp[j] == 0)
			continue;
		GemmSeg s {};
		s.a_off = mp.bs_off[j] / 32;
		s.lda   = int(mp.Mp[j]);
		s.b_off = mp.xs_off[j] / 32;
		s.ldb   = int(round8(plan.l[j]));
		s.K     = int(round32(plan.r[j]));
		s.dep   = int(j);
		const int sb = int(mp.seg1.size());
		mp.seg1.push_back(s);
		add_tc_tiles(mp.tile1, mp.bxs_off[j], mp.Mp[j], mp.Mp[j], plan.l[j], sb, sb + 1, mp.bm, bn);
	}
	// pass 2: C = Y_i (FP64, column-major)
	size_t t = 0;
	for (size_t i = 0; i < np; ++i) {
		const int sb = int(mp.seg2.size());
		for (; t < nt && plan.triples[t].i == int(i); ++t) {
			const Triple& tr = plan.triples[t];
			GemmSeg       s {};
			s.a_off = mp.bxs_off[tr.j] / 32 + mp.group_row[t];
			s.lda   = int(mp.Mp[tr.j]);
			s.b_off = mp.at_off[t] / 32;
			s.ldb   = int(round8(plan.l[i]));
			s.K     = int(round32(plan.l[tr.j]));
			s.dep   = tr.j;
			mp.seg2.push_back(s);
		}
		add_tc_tiles(mp.tile2, plan.xy_start[i], plan.r[i], plan.r[i], plan.l[i], sb,
		             int(mp.seg2.size()), mp.bm, bn);
	}
	auto kcost = [](const std::vector<GemmSeg>& segs, const GemmTile& g) {
		long long k = 0;
		for (int s = g.seg_begin; s < g.seg_end; ++s)
			k += segs[s].K;
		return k;
	};
	// split long pass-2 tiles along K (whole segments per part) so that the
	// pass has about two parts per SM; a part keeps at least 16 k-chunks (the
	// partial-tile round trip and the final reduction cost about that much)
	{
		long long total = 0;
		for (const GemmTile& g : mp.tile2)
			total += kcost(mp.seg2, g) / 32;
		const long long target = std::max<long long>(16, total / (2LL * std::max(sms, 1)));
		std::vector<GemmTile> out;
		for (const GemmTile& g : mp.tile2) {
			const long long c = kcost(mp.seg2, g) / 32;
			if (c <= 2 * target || g.seg_end - g.seg_begin < 2) {
				out.push_back(g);
				continue;
			}
			std::vector<std::pair<int, int>> parts;
			int       b   = g.seg_begin;
			long long acc = 0;
			for (int q = g.seg_begin; q < g.seg_end; ++q) {
				acc += mp.seg2[size_t(q)].K / 32;
				if (acc >= target && q + 1 < g.seg_end) {
					parts.push_back({ b, q + 1 });
					b   = q + 1;
					acc = 0;
				}
			}
			parts.push_back({ b, g.seg_end });
			if (parts.size() < 2) {
				out.push_back(g);
				continue;
			}
			const int tile_id = mp.n_split_tiles++;
			for (size_t q = 0; q < parts.size(); ++q) {
				GemmTile part   = g;
				part.seg_begin  = parts[q].first;
				part.seg_end    = parts[q].second;
				part.nsplit     = int(parts.size());
				part.split_part = int(q);
				part.split_tile = tile_id;
				part.slot       = int(mp.split_slots);
				out.push_back(part);
			}
			mp.split_slots += (long long)parts.size();
		}
		mp.tile2.swap(out);
	}
	std::stable_sort(mp.tile1.begin(), mp.tile1.end(), [&](const GemmTile& x, const GemmTile& y) {
		return kcost(mp.seg1, x) > kcost(mp.seg1, y);
	});
	std::stable_sort(mp.tile2.begin(), mp.tile2.end(), [&](const GemmTile& x, const GemmTile& y) {
		return kcost(mp.seg2, x) > kcost(mp.seg2, y);
	});
	return std::string();
}

int balance_tiles(std::vector<GemmTile>& tiles, const std::vector<GemmSeg>& segs, int bins,
                  std::vector<int>& starts)
{
	const int n = int(tiles.size());
	const int G = std::max(1, std::min(bins, n));
	std::vector<long long> cost(size_t(n), 0);
	for (int t = 0; t < n; ++t) {
		long long c = 2;
		for (int s = tiles[size_t(t)].seg_begin; s < tiles[size_t(t)].seg_end; ++s)
			c += segs[size_t(s)].K / 32;
		cost[size_t(t)] = c;
	}
	std::vector<int> order(static_cast<size_t>(n));
	std::iota(order.begin(), order.end(), 0);
	std::stable_sort(order.begin(), order.end(),
	                 [&](int a, int b) { return cost[size_t(a)] > cost[size_t(b)]; });
	// min-heap of (load, bin)
	std::vector<std::pair<long long, int>> heap;
	for (int b = 0; b < G; ++b)
		heap.push_back({0, b});
	auto cmp = [](const std::pair<long long, int>& x, const std::pair<long long, int>& y) {
		return x.first != y.first ? x.first > y.first : x.second > y.second;
	};
	std::make_heap(heap.begin(), heap.end(), cmp);
	std::vector<std::vector<int>> runs(static_cast<size_t>(G));
	for (int t : order) {
		std::pop_heap(heap.begin(), heap.end(), cmp);
		auto& top = heap.back();
		runs[size_t(top.second)].push_back(t);
		top.first += cost[size_t(t)];
		std::push_heap(heap.begin(), heap.end(), cmp);
	}
	std::vector<GemmTile> out;
	out.reserve(size_t(n));
	starts.assign(size_t(G) + 1, 0);
	for (int b = 0; b < G; ++b) {
		starts[size_t(b)] = int(out.size());
		for (int t : runs[size_t(b)])
			out.push_back(tiles[size_t(t)]);
	}
	starts[size_t(G)] = int(out.size());
	tiles.swap(out);
	return n == 0 ? 0 : G;
}

std::vector<PackJob> mixed_pack_jobs(const KronPlan& P)
{
	const MixedPlan&     mp = P.mixed;
	std::vector<PackJob> jobs;
	jobs.reserve(2 * P.triples.size());
	for (size_t t = 0; t < P.triples.size(); ++t) {
		const Triple& tr = P.triples[t];
		const size_t  i = size_t(tr.i), j = size_t(tr.j);
		// B_k(i,j): rows row_off of Bstack_j (M_j x r_j) -> rows group_row of the chunked Bstack_j
		jobs.push_back({ P.bstack_off[j] + P.row_off[t], mp.bs_off[j], int(P.M[j]), int(P.r[i]),
		                 int(P.r[j]), int(mp.Mp[j]), int(mp.group_row[t]), 0 });
		// A_k(i,j)^T (l_j x l_i, ld l_j) -> rows l_i, K = l_j of the chunked A^T block
		jobs.push_back({ P.at_off[t], mp.at_off[t], int(P.l[j]), int(P.l[j]), int(P.l[i]),
		                 int(round8(P.l[i])), 0, 1 });
	}
	return jobs;
}

} // namespace dmrgpp

