// Host emulation of a group (many independent sectors in one persistent
// launch, dmrgpp_kron_create_group) over the work list that
// collect_triples + build_kron_plan_triples + build_persistent_schedule
// produce.  Each work item belongs to a sector (a pass-1 item to its input
// patch's, a pass-2 item to its output's), and the masked group solvers skip
// the items of stopped sectors.  Checks, on the CPU, that this is safe:
//   * every pass-2 segment depends on a patch of the item's own sector, and
//     every operand load stays inside that sector's x and BX;
//   * with any one sector stopped (its items skipped, its x set to NaN) the
//     other sectors' results equal their own H*x and the stopped sector's
//     output is left as it was; with none stopped, every sector's result is
//     its own H*x.
// Usage: group_schedule_check seed nsectors max_patches max_terms max_size
// Prints "ok <max relative error> <items>" or "FAIL <reason>" (exit code 1).
#include "kron_plan.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <map>
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
	if (argc < 6)
		return fail("usage");
	const unsigned seed = unsigned(std::atoi(argv[1]));
	const int      nsec = std::atoi(argv[2]);
	const int      maxp = std::atoi(argv[3]);
	const int      maxk = std::atoi(argv[4]);
	const int      maxs = std::atoi(argv[5]);
	std::mt19937_64                        rng(seed);
	std::uniform_real_distribution<double> val(-1.0, 1.0);
	std::uniform_real_distribution<double> coin(0.0, 1.0);
	auto uni = [&](int a, int b) { return std::uniform_int_distribution<int>(a, b)(rng); };

	std::vector<std::vector<double>> store;
	std::vector<size_t>              l, r;
	std::vector<Triple>              triples;
	std::vector<BlockRef>            blocks;
	std::vector<long long>           starts(1, 0);
	std::vector<int>                 patch_sector;
	double                           f_alg = 0.0;
	size_t                           nop   = 0;
	store.reserve(100000);
	for (int s = 0; s < nsec; ++s) {
		const int           np = uni(1, maxp), nk = uni(1, maxk);
		std::vector<size_t> ls(static_cast<size_t>(np)), rs(static_cast<size_t>(np));
		for (int p = 0; p < np; ++p)
			ls[size_t(p)] = size_t(uni(1, maxs)), rs[size_t(p)] = size_t(uni(1, maxs));
		const size_t               nt = size_t(np) * size_t(np) * size_t(nk);
		std::vector<const double*> A(nt, nullptr), B(nt, nullptr);
		std::vector<size_t>        ldA(nt, 0), ldB(nt, 0);
		for (int k = 0; k < nk; ++k)
			for (int j = 0; j < np; ++j)
				for (int i = 0; i < np; ++i) {
					if (coin(rng) < 0.4)
						continue;
					const size_t ix = size_t(i) + size_t(j) * size_t(np) + size_t(k) * size_t(np) * size_t(np);
					ldA[ix]         = ls[size_t(i)];
					ldB[ix]         = rs[size_t(i)] + (coin(rng) < 0.3 ? 1 : 0);
					store.emplace_back(ldA[ix] * ls[size_t(j)]);
					for (double& v : store.back())
						v = val(rng);
					A[ix] = store.back().data();
					store.emplace_back(ldB[ix] * rs[size_t(j)]);
					for (double& v : store.back())
						v = val(rng);
					B[ix] = store.back().data();
				}
		const std::string msg = collect_triples(size_t(nk), size_t(np), ls.data(), rs.data(), A.data(), ldA.data(),
		                                        B.data(), ldB.data(), int(l.size()), triples, blocks, f_alg);
		if (!msg.empty())
			return fail(msg.c_str(), s, 0);
		long long dim = 0;
		for (int p = 0; p < np; ++p) {
			l.push_back(ls[size_t(p)]);
			r.push_back(rs[size_t(p)]);
			patch_sector.push_back(s);
			dim += (long long)(ls[size_t(p)] * rs[size_t(p)]);
		}
		starts.push_back(starts.back() + dim);
		nop = std::max(nop, size_t(nk));
	}
	KronPlan          plan;
	PackBuffer        pack;
	const std::string msg = build_kron_plan_triples(nop, l.size(), l.data(), r.data(), triples, blocks, f_alg, 64, 64,
	                                                plan, &pack);
	if (!msg.empty())
		return fail(msg.c_str());
	const long long dim = plan.dim();
	if (dim != starts.back())
		return fail("union dimension", dim, starts.back());
	auto sector_of = [&](long long off) {
		return int(std::upper_bound(starts.begin(), starts.end(), off) - starts.begin()) - 1;
	};
	std::vector<double> x(static_cast<size_t>(dim));
	for (double& v : x)
		v = val(rng);
	std::vector<double> yref(static_cast<size_t>(dim), 0.0);
	for (size_t t = 0; t < plan.triples.size(); ++t) {
		const Triple&       tr = plan.triples[t];
		const BlockRef&     bl = plan.blocks[t];
		if (patch_sector[size_t(tr.i)] != patch_sector[size_t(tr.j)])
			return fail("triple couples two sectors", tr.i, tr.j);
		const long long     ri = plan.r[size_t(tr.i)], li = plan.l[size_t(tr.i)];
		const long long     rj = plan.r[size_t(tr.j)], lj = plan.l[size_t(tr.j)];
		const double*       X  = x.data() + plan.xy_start[size_t(tr.j)];
		double*             Y  = yref.data() + plan.xy_start[size_t(tr.i)];
		std::vector<double> T(size_t(ri * lj), 0.0);
		for (long long c = 0; c < lj; ++c)
			for (long long q = 0; q < rj; ++q)
				for (long long a = 0; a < ri; ++a)
					T[size_t(a + c * ri)] += bl.B[a + q * (long long)bl.ldB] * X[q + c * rj];
		for (long long n = 0; n < li; ++n)
			for (long long c = 0; c < lj; ++c)
				for (long long a = 0; a < ri; ++a)
					Y[a + n * ri] += T[size_t(a + c * ri)] * bl.A[n + c * (long long)bl.ldA];
	}
	std::vector<double> yscale(static_cast<size_t>(nsec), 1e-300);
	for (long long e = 0; e < dim; ++e)
		yscale[size_t(sector_of(e))] = std::max(yscale[size_t(sector_of(e))], std::fabs(yref[size_t(e)]));

	const int tiles[] = { 32, 64 }, bks[] = { 16, 64 }, grids[] = { 7, 296 };
	double    worst = 0.0;
	size_t    items = 0;
	for (int tile : tiles)
		for (int bk : bks)
			for (int grid : grids) {
				build_tile_lists(plan, tile, tile);
				build_persistent_schedule(plan, bk, grid, 2);
				const std::string verdict = validate_persistent_schedule(plan, tile);
				if (!verdict.empty())
					return fail(("the validator rejects a good group schedule: " + verdict).c_str());
				const auto&      W = plan.items;
				std::vector<int> sec(W.size());
				for (size_t q = 0; q < W.size(); ++q) // as the group handle assigns them
					sec[q] = W[q].kind == 0 ? sector_of(plan.xy_start[size_t(W[q].producer)]) : sector_of(W[q].c_off);
				for (size_t q = size_t(plan.n1_items); q < W.size(); ++q)
					for (int e = W[q].seg_begin; e < W[q].seg_end; ++e)
						if (patch_sector[size_t(plan.pseg2[size_t(e)].dep)] != sec[q])
							return fail("pass-2 segment depends on another sector", (long long)q, e);
				for (int stopped = -1; stopped < nsec; ++stopped) {
					items += W.size();
					const double nan = std::numeric_limits<double>::quiet_NaN();
					std::vector<double> xin(x);
					for (long long e = 0; e < dim; ++e)
						if (sector_of(e) == stopped)
							xin[size_t(e)] = nan;
					std::vector<double> bx(size_t(std::max<long long>(plan.bx_elems, 1)), nan);
					std::vector<double> y(static_cast<size_t>(dim), -7.0);
					std::map<long long, std::vector<double>> slot;
					std::map<int, const KronItem*>           split_head;
					for (size_t q = 0; q < W.size(); ++q) {
						if (sec[q] == stopped)
							continue;
						const KronItem&             w    = W[q];
						const std::vector<GemmSeg>& segs = w.kind == 0 ? plan.seg1 : plan.pseg2;
						std::vector<double>         part(size_t(tile) * size_t(tile), 0.0);
						for (int n = w.n0; n < std::min(w.n0 + tile, w.N); ++n)
							for (int m = w.m0; m < std::min(w.m0 + tile, w.M); ++m) {
								double s = 0.0;
								for (int e = w.seg_begin; e < w.seg_end; ++e) {
									const GemmSeg& g = segs[size_t(e)];
									for (int k = 0; k < g.K; ++k) {
										const long long ia = g.a_off + m + (long long)k * g.lda;
										const long long ib = g.b_off + k + (long long)n * g.ldb;
										if (w.kind == 0) {
											if (ib < starts[size_t(sec[q])] || ib >= starts[size_t(sec[q]) + 1])
												return fail("pass-1 x load outside the sector", (long long)q, ib);
											s += pack[size_t(ia)] * xin[size_t(ib)];
										} else {
											const long long lo = plan.bx_off[size_t(g.dep)],
											                hi = lo + plan.M[size_t(g.dep)] * plan.l[size_t(g.dep)];
											if (ia < lo || ia >= hi)
												return fail("pass-2 BX load outside its dependency", (long long)q, ia);
											s += bx[size_t(ia)] * pack[size_t(ib)];
										}
									}
								}
								const long long ic = w.c_off + m + (long long)n * w.ldc;
								if (w.kind == 0)
									bx[size_t(ic)] = s;
								else if (w.kind == 1)
									y[size_t(ic)] = s;
								else
									part[size_t(m - w.m0) + size_t(n - w.n0) * size_t(tile)] = s;
							}
						if (w.kind == 2) {
							slot[w.slot + w.part] = part;
							split_head[w.tile]    = &w;
						}
					}
					for (const auto& kv : split_head) {
						const KronItem& w0 = *kv.second;
						for (int n = w0.n0; n < std::min(w0.n0 + tile, w0.N); ++n)
							for (int m = w0.m0; m < std::min(w0.m0 + tile, w0.M); ++m) {
								double s = 0.0;
								for (int p = 0; p < w0.nsplit; ++p)
									s += slot[w0.slot + p][size_t(m - w0.m0) + size_t(n - w0.n0) * size_t(tile)];
								y[size_t(w0.c_off + m + (long long)n * w0.ldc)] = s;
							}
					}
					for (long long e = 0; e < dim; ++e) {
						const int sc = sector_of(e);
						if (sc == stopped) {
							if (y[size_t(e)] != -7.0)
								return fail("stopped sector's output written", stopped, e);
							continue;
						}
						const double d = std::fabs(y[size_t(e)] - yref[size_t(e)]) / yscale[size_t(sc)];
						if (!(d <= 1e-12))
							return fail("sector result differs from its H*x", sc, e);
						worst = std::max(worst, d);
					}
				}
			}
	std::printf("ok %.3e %zu\n", worst, items);
	return 0;
}
