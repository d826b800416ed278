// Host planning and packing of the patch-wise wave-function transformation
// (wft_plan.h).
#include "wft_plan.h"

#include <algorithm>
#include <climits>

namespace dmrgpp {

namespace {

constexpr long long kAlign = 32; // doubles between packed blocks

long long align_up(long long x) { return (x + kAlign - 1) / kAlign * kAlign; }

void tiles_of(std::vector<GemmTile>& tiles, long long c_off, long long ldc, long long M, long long N,
              int seg_begin, int seg_end, int bm, int bn)
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

} // namespace

std::string build_wft_plan(const dmrgpp_wft_desc& d, WftPlan& plan, std::vector<double>* packed)
{
	plan = WftPlan();
	if (d.np_in == 0 || d.np_out == 0)
		return "np_in and np_out must be >= 1";
	if (!d.l_in || !d.r_in || !d.l_out || !d.r_out || !d.src || !d.WL || !d.ld_WL || !d.WR || !d.ld_WR)
		return "null table or size array";
	plan.np_in  = d.np_in;
	plan.np_out = d.np_out;
	plan.x_start.assign(d.np_in + 1, 0);
	plan.y_start.assign(d.np_out + 1, 0);
	long long maxs = 0;
	for (size_t p = 0; p < d.np_in; ++p) {
		if (d.l_in[p] < 1 || d.r_in[p] < 1 || d.l_in[p] > size_t(INT_MAX) || d.r_in[p] > size_t(INT_MAX))
			return "input patch " + std::to_string(p) + " has an empty or oversized group";
		plan.l_in.push_back((long long)d.l_in[p]);
		plan.r_in.push_back((long long)d.r_in[p]);
		plan.x_start[p + 1] = plan.x_start[p] + plan.l_in[p] * plan.r_in[p];
		maxs                = std::max({ maxs, plan.l_in[p], plan.r_in[p] });
	}
	for (size_t q = 0; q < d.np_out; ++q) {
		if (d.l_out[q] < 1 || d.r_out[q] < 1 || d.l_out[q] > size_t(INT_MAX) || d.r_out[q] > size_t(INT_MAX))
			return "output patch " + std::to_string(q) + " has an empty or oversized group";
		plan.l_out.push_back((long long)d.l_out[q]);
		plan.r_out.push_back((long long)d.r_out[q]);
		plan.y_start[q + 1] = plan.y_start[q] + plan.l_out[q] * plan.r_out[q];
		maxs                = std::max({ maxs, plan.l_out[q], plan.r_out[q] });
		const long long p   = d.src[q];
		if (p >= (long long)d.np_in)
			return "output patch " + std::to_string(q) + ": source patch out of range";
		plan.src.push_back(p < 0 ? -1 : p);
		if (p < 0)
			continue;
		if (!d.WL[q] || !d.WR[q])
			return "output patch " + std::to_string(q) + ": null transformation block";
		// stored rows of each block (transposed storage swaps the dimensions)
		const size_t wl_rows = d.trans_WL ? d.l_in[p] : d.l_out[q];
		const size_t wr_rows = d.trans_WR ? d.r_in[p] : d.r_out[q];
		if (d.ld_WL[q] < wl_rows || d.ld_WR[q] < wr_rows)
			return "output patch " + std::to_string(q) + ": leading dimension smaller than the block's rows";
	}
	if (plan.x_start.back() > (long long)INT_MAX * 64 || plan.y_start.back() > (long long)INT_MAX * 64)
		return "sector too large";
	plan.bm = plan.bn = maxs > 192 ? 64 : 32;

	// packed blocks and the intermediate T
	plan.wr_off.assign(d.np_out, 0);
	plan.wlt_off.assign(d.np_out, 0);
	plan.t_off.assign(d.np_out, 0);
	long long off = 0, toff = 0;
	for (size_t q = 0; q < d.np_out; ++q) {
		const long long p = plan.src[q];
		if (p < 0)
			continue;
		plan.wr_off[q] = off;
		off += align_up(plan.r_out[q] * plan.r_in[p]);
		plan.wlt_off[q] = off;
		off += align_up(plan.l_in[p] * plan.l_out[q]);
		plan.t_off[q] = toff;
		toff += align_up(plan.r_out[q] * plan.l_in[p]);
		plan.flops += 2.0 * double(plan.r_out[q]) * double(plan.l_in[p])
		    * (double(plan.r_in[p]) + double(plan.l_out[q]));
	}
	plan.op_elems = off;
	plan.t_elems  = toff;

	if (packed) {
		packed->assign(size_t(std::max<long long>(off, 1)), 0.0);
		double* P = packed->data();
		parallel_for(d.np_out, [&](size_t q) {
			const long long p = plan.src[q];
			if (p < 0)
				return;
			const long long ro = plan.r_out[q], ri = plan.r_in[p], li = plan.l_in[p], lo = plan.l_out[q];
			// WR_q as r_out x r_in, column-major (ld r_out)
			double*       wr  = P + plan.wr_off[q];
			const double* swr = d.WR[q];
			const long long lwr = (long long)d.ld_WR[q];
			for (long long c = 0; c < ri; ++c)
				for (long long a = 0; a < ro; ++a)
					wr[a + c * ro] = d.trans_WR ? swr[c + a * lwr] : swr[a + c * lwr];
			// WL_q^T as l_in x l_out, column-major (ld l_in): element (k, n) = WL(n, k)
			double*       wlt = P + plan.wlt_off[q];
			const double* swl = d.WL[q];
			const long long lwl = (long long)d.ld_WL[q];
			for (long long n = 0; n < lo; ++n)
				for (long long k = 0; k < li; ++k)
					wlt[k + n * li] = d.trans_WL ? swl[k + n * lwl] : swl[n + k * lwl];
		});
	}

	// pass A: T_q = WR_q (r_out x r_in) * X_p (r_in x l_in)
	for (size_t q = 0; q < d.np_out; ++q) {
		const long long p = plan.src[q];
		if (p < 0)
			continue;
		GemmSeg s {};
		s.a_off = plan.wr_off[q];
		s.lda   = int(plan.r_out[q]);
		s.b_off = plan.x_start[p];
		s.ldb   = int(plan.r_in[p]);
		s.K     = int(plan.r_in[p]);
		s.dep   = int(p);
		const int sb = int(plan.segA.size());
		plan.segA.push_back(s);
		tiles_of(plan.tileA, plan.t_off[q], plan.r_out[q], plan.r_out[q], plan.l_in[p], sb, sb + 1,
		         plan.bm, plan.bn);
	}
	// pass B: Y_q = T_q (r_out x l_in) * WL_q^T (l_in x l_out); no source: zeros
	for (size_t q = 0; q < d.np_out; ++q) {
		const long long p  = plan.src[q];
		const int       sb = int(plan.segB.size());
		if (p >= 0) {
			GemmSeg s {};
			s.a_off = plan.t_off[q];
			s.lda   = int(plan.r_out[q]);
			s.b_off = plan.wlt_off[q];
			s.ldb   = int(plan.l_in[p]);
			s.K     = int(plan.l_in[p]);
			s.dep   = int(p);
			plan.segB.push_back(s);
		}
		tiles_of(plan.tileB, plan.y_start[q], plan.r_out[q], plan.r_out[q], plan.l_out[q], sb,
		         int(plan.segB.size()), plan.bm, plan.bn);
	}
	return std::string();
}

} // namespace dmrgpp
