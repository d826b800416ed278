// Host emulation of the patch-wise wave-function transformation plan
// (build_wft_plan, wft_plan.h): replays the two grouped GEMM passes from the
// plan's segment and tile lists and the packed blocks exactly as the grouped
// DGEMM kernel reads them (kron_gemm.cu: A M-contiguous, B K-contiguous,
// C column-major), checks that every read and write stays inside its buffer
// and that every output element is written once, and compares the result
// with Y_q = WR_q X_p WL_q^T computed directly from the caller's blocks.
// Usage: wft_plan_check seed np_in np_out max_size trans_WL trans_WR
// Prints "ok <max relative error>" or "FAIL <reason>" (exit code 1).
#include "wft_plan.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

using namespace dmrgpp;

namespace {

int fail(const char* why, long long a = 0, long long b = 0)
{
	std::printf("FAIL %s %lld %lld\n", why, a, b);
	return 1;
}

} // namespace

int main(int argc, char** argv)
{
	if (argc < 7)
		return fail("usage");
	const unsigned seed = unsigned(std::atoi(argv[1]));
	const int      npi  = std::atoi(argv[2]);
	const int      npo  = std::atoi(argv[3]);
	const int      maxs = std::atoi(argv[4]);
	const int      tl   = std::atoi(argv[5]);
	const int      tr   = std::atoi(argv[6]);
	std::mt19937_64                        rng(seed);
	std::uniform_int_distribution<int>     size(1, maxs);
	std::uniform_real_distribution<double> val(-1.0, 1.0);
	std::uniform_real_distribution<double> coin(0.0, 1.0);

	std::vector<size_t> li(npi), ri(npi), lo(npo), ro(npo), ldwl(npo, 0), ldwr(npo, 0);
	std::vector<long long> src(npo);
	for (int p = 0; p < npi; ++p) {
		li[p] = size_t(size(rng));
		ri[p] = size_t(size(rng));
	}
	std::vector<std::vector<double>> WLs(npo), WRs(npo);
	std::vector<const double*>       WL(npo, nullptr), WR(npo, nullptr);
	for (int q = 0; q < npo; ++q) {
		lo[q]  = size_t(size(rng));
		ro[q]  = size_t(size(rng));
		src[q] = coin(rng) < 0.15 ? -1 : (long long)(rng() % npi);
		if (src[q] < 0)
			continue;
		const size_t p = size_t(src[q]);
		// stored dimensions (transposed storage swaps them) and padded ld
		const size_t wl_rows = tl ? li[p] : lo[q], wl_cols = tl ? lo[q] : li[p];
		const size_t wr_rows = tr ? ri[p] : ro[q], wr_cols = tr ? ro[q] : ri[p];
		ldwl[q] = wl_rows + (coin(rng) < 0.3 ? 2 : 0);
		ldwr[q] = wr_rows + (coin(rng) < 0.3 ? 3 : 0);
		WLs[q].resize(ldwl[q] * wl_cols);
		WRs[q].resize(ldwr[q] * wr_cols);
		for (double& v : WLs[q])
			v = val(rng);
		for (double& v : WRs[q])
			v = val(rng);
		WL[q] = WLs[q].data();
		WR[q] = WRs[q].data();
	}
	dmrgpp_wft_desc d {};
	d.np_in    = size_t(npi);
	d.l_in     = li.data();
	d.r_in     = ri.data();
	d.np_out   = size_t(npo);
	d.l_out    = lo.data();
	d.r_out    = ro.data();
	d.src      = src.data();
	d.WL       = WL.data();
	d.ld_WL    = ldwl.data();
	d.WR       = WR.data();
	d.ld_WR    = ldwr.data();
	d.trans_WL = tl;
	d.trans_WR = tr;
	d.device   = -1;
	WftPlan             plan;
	std::vector<double> packed;
	const std::string   msg = build_wft_plan(d, plan, &packed);
	if (!msg.empty())
		return fail(msg.c_str());
	const long long Din = plan.dim_in(), Dout = plan.dim_out();
	std::vector<double> x(static_cast<size_t>(Din));
	for (double& v : x)
		v = val(rng);

	// one grouped pass: C tiles = sum over segments of A(M x K) * B(K x N)
	auto pass = [&](const std::vector<GemmSeg>& segs, const std::vector<GemmTile>& tiles,
	                const std::vector<double>& A, const std::vector<double>& B, std::vector<double>& C,
	                std::vector<int>& hits) -> int {
		for (const GemmTile& t : tiles) {
			for (int m = t.m0; m < std::min(t.M, t.m0 + plan.bm); ++m)
				for (int n = t.n0; n < std::min(t.N, t.n0 + plan.bn); ++n) {
					double s = 0.0;
					for (int g = t.seg_begin; g < t.seg_end; ++g) {
						const GemmSeg& sg = segs[size_t(g)];
						for (int k = 0; k < sg.K; ++k) {
							const long long ia = sg.a_off + (long long)k * sg.lda + m;
							const long long ib = sg.b_off + (long long)n * sg.ldb + k;
							if (ia < 0 || ia >= (long long)A.size() || ib < 0 || ib >= (long long)B.size())
								return fail("operand read out of bounds", ia, ib);
							s += A[size_t(ia)] * B[size_t(ib)];
						}
					}
					const long long ic = t.c_off + (long long)n * t.ldc + m;
					if (ic < 0 || ic >= (long long)C.size())
						return fail("store out of bounds", ic, (long long)C.size());
					C[size_t(ic)] = s;
					++hits[size_t(ic)];
				}
		}
		return 0;
	};
	std::vector<double> T(static_cast<size_t>(std::max<long long>(plan.t_elems, 1)), 0.0),
	    y(static_cast<size_t>(Dout), 0.0);
	std::vector<int>    hitT(T.size(), 0), hitY(y.size(), 0);
	if (pass(plan.segA, plan.tileA, packed, x, T, hitT) || pass(plan.segB, plan.tileB, T, packed, y, hitY))
		return 1;
	for (long long e = 0; e < Dout; ++e)
		if (hitY[size_t(e)] != 1)
			return fail("output element not written exactly once", e, hitY[size_t(e)]);

	// direct: Y_q (ro x lo) = WR (ro x ri) * X_p (ri x li) * WL^T (li x lo)
	double err = 0.0, ref = 0.0;
	for (int q = 0; q < npo; ++q) {
		const long long y0 = plan.y_start[size_t(q)];
		for (size_t a = 0; a < ro[q]; ++a)
			for (size_t b = 0; b < lo[q]; ++b) {
				double s = 0.0;
				if (src[q] >= 0) {
					const size_t    p  = size_t(src[q]);
					const long long x0 = plan.x_start[p];
					for (size_t c = 0; c < ri[p]; ++c)
						for (size_t k = 0; k < li[p]; ++k) {
							const double wr = tr ? WR[q][c + a * ldwr[q]] : WR[q][a + c * ldwr[q]];
							const double wl = tl ? WL[q][k + b * ldwl[q]] : WL[q][b + k * ldwl[q]];
							s += wr * x[size_t(x0 + (long long)c + (long long)k * (long long)ri[p])] * wl;
						}
				}
				const double got = y[size_t(y0 + (long long)a + (long long)b * (long long)ro[q])];
				err = std::max(err, std::fabs(got - s));
				ref = std::max(ref, std::fabs(s));
			}
	}
	const double rel = ref > 0 ? err / ref : err;
	if (!(rel < 1e-12))
		return fail("result differs from the direct product", (long long)(rel * 1e15), 0);
	std::printf("ok %.3e flops %.0f\n", rel, plan.flops);
	return 0;
}
