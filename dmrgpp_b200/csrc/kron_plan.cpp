// Host-side planning of the two grouped-GEMM passes (see kron_plan.h).
#include "kron_plan.h"

#include <algorithm>
#include <climits>
#include <numeric>

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
                            std::vector<double>* pack_host)
{
	if (noperator == 0 || npatches == 0)
		return "noperator and npatches must be >= 1";
	if (!lsz || !rsz || !A || !ldA || !B || !ldB)
		return "null table or size array";
	const size_t np = npatches;
	const size_t np2 = np * np;
	plan     = KronPlan();
	plan.np  = np;
	plan.nop = noperator;
	plan.bm  = bm;
	plan.bn  = bn;
	plan.l.resize(np);
	plan.r.resize(np);
	plan.xy_start.assign(np + 1, 0);
	for (size_t p = 0; p < np; ++p) {
		// the reference asserts 1 <= size (setup_sparse_batch.cpp:70-71)
		if (lsz[p] < 1 || rsz[p] < 1)
			return "patch " + std::to_string(p) + " has an empty left or right group";
		if (lsz[p] > INT_MAX / 64 || rsz[p] > INT_MAX / 64)
			return "patch " + std::to_string(p) + " is too large";
		plan.l[p]            = (long long)lsz[p];
		plan.r[p]            = (long long)rsz[p];
		plan.xy_start[p + 1] = plan.xy_start[p] + plan.l[p] * plan.r[p];
	}

	// contributing triples (setup_nC.cpp:43-121): both blocks present and
	// each with at least one nonzero entry
	for (size_t i = 0; i < np; ++i)
		for (size_t j = 0; j < np; ++j)
			for (size_t k = 0; k < noperator; ++k) {
				const size_t t = i + j * np + k * np2;
				if (!A[t] || !B[t])
					continue;
				if (ldA[t] < lsz[i] || ldB[t] < rsz[i])
					return "leading dimension smaller than the block's rows at table entry "
					    + std::to_string(t);
				if (!has_nonzero(A[t], ldA[t], lsz[i], lsz[j])
				    || !has_nonzero(B[t], ldB[t], rsz[i], rsz[j]))
					continue;
				plan.triples.push_back({ int(i), int(j), int(k) });
				plan.f_alg += 2.0 * double(rsz[i]) * double(lsz[j])
				    * (double(rsz[j]) + double(lsz[i]));
			}

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
		pack_host->assign(size_t(plan.op_elems), 0.0);
		double* P = pack_host->data();
		for (size_t t = 0; t < nt; ++t) {
			const Triple& tr = plan.triples[t];
			const size_t  ix = size_t(tr.i) + size_t(tr.j) * np + size_t(tr.k) * np2;
			// B_k(i,j) (r_i x r_j) into rows [row_off, row_off + r_i) of Bstack_j
			const long long Mj = plan.M[tr.j];
			double*         bs = P + plan.bstack_off[tr.j] + plan.row_off[t];
			const double*   b  = B[ix];
			for (long long c = 0; c < plan.r[tr.j]; ++c)
				for (long long q = 0; q < plan.r[tr.i]; ++q)
					bs[q + c * Mj] = b[q + c * (long long)ldB[ix]];
			// A_k(i,j)^T (l_j x l_i), leading dimension l_j
			double*         at = P + plan.at_off[t];
			const double*   a  = A[ix];
			const long long lj = plan.l[tr.j];
			for (long long c = 0; c < plan.l[tr.i]; ++c)
				for (long long q = 0; q < lj; ++q)
					at[q + c * lj] = a[c + q * (long long)ldA[ix]];
		}
	}

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
			plan.seg2.push_back(s);
		}
		const int se = int(plan.seg2.size());
		add_tiles(plan.tile2, plan.xy_start[i], plan.r[i], plan.r[i], plan.l[i], sb, se, bm, bn);
	}
	order_tiles(plan.tile2, plan.seg2);
	return std::string();
}

} // namespace dmrgpp
