// Host emulation of the persistent FP64 H*x launch (kron_persistent.cu)
// over the work list that build_tile_lists + build_persistent_schedule
// produce, for every tile shape and K-chunk of the launch configurations
// and a range of grid sizes.  Checks, on the CPU, what the kernel relies on:
//   * pass-1 items come first, one per tile of BX_j = Bstack_j X_j, and
//     n1_of_j counts them; every pass-2 item holds at most kMaxItemSegs
//     segments, and its first segment is copied into seg0;
//   * every operand element an item loads lies inside its buffer (packed
//     operators, x, BX), and a pass-2 segment reads only BX rows of the
//     input patch it names as its dependency, every one of them written by
//     that patch's pass-1 items (the kernel waits on exactly those);
//   * every BX and every Y element is written exactly once, split tiles
//     through their partial slots summed in part order;
//   * the result equals H*x computed directly from the caller's blocks;
//   * validate_persistent_schedule (the library's debug-mode check) accepts
//     every schedule and rejects spoilt copies of one.
// Usage: persistent_schedule_check seed npatches noperator max_size
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
	if (argc < 5)
		return fail("usage");
	const unsigned seed = unsigned(std::atoi(argv[1]));
	const int      np   = std::atoi(argv[2]);
	const int      nop  = std::atoi(argv[3]);
	const int      maxs = std::atoi(argv[4]);
	std::mt19937_64                        rng(seed);
	std::uniform_int_distribution<int>     size(1, maxs);
	std::uniform_real_distribution<double> val(-1.0, 1.0);
	std::uniform_real_distribution<double> coin(0.0, 1.0);

	std::vector<size_t> l(static_cast<size_t>(np)), r(static_cast<size_t>(np));
	for (int p = 0; p < np; ++p) {
		l[size_t(p)] = size_t(size(rng));
		r[size_t(p)] = size_t(size(rng));
	}
	const size_t                     nt = size_t(np) * size_t(np) * size_t(nop);
	std::vector<std::vector<double>> Ast(nt), Bst(nt);
	std::vector<const double*>       A(nt, nullptr), B(nt, nullptr);
	std::vector<size_t>              ldA(nt, 0), ldB(nt, 0);
	for (int k = 0; k < nop; ++k)
		for (int j = 0; j < np; ++j)
			for (int i = 0; i < np; ++i) {
				if (coin(rng) < 0.4)
					continue;
				const size_t ix = size_t(i) + size_t(j) * size_t(np) + size_t(k) * size_t(np) * size_t(np);
				ldA[ix]         = l[size_t(i)] + (coin(rng) < 0.3 ? 2 : 0);
				ldB[ix]         = r[size_t(i)] + (coin(rng) < 0.3 ? 3 : 0);
				Ast[ix].resize(ldA[ix] * l[size_t(j)]);
				Bst[ix].resize(ldB[ix] * r[size_t(j)]);
				for (double& v : Ast[ix])
					v = val(rng);
				for (double& v : Bst[ix])
					v = val(rng);
				A[ix] = Ast[ix].data();
				B[ix] = Bst[ix].data();
			}
	KronPlan          plan;
	PackBuffer        pack;
	const std::string msg = build_kron_plan(size_t(nop), size_t(np), l.data(), r.data(), A.data(), ldA.data(),
	                                        B.data(), ldB.data(), 64, 64, plan, &pack);
	if (!msg.empty())
		return fail(msg.c_str());
	const long long     dim = plan.dim();
	std::vector<double> x(static_cast<size_t>(dim));
	for (double& v : x)
		v = val(rng);
	// direct H*x from the caller's blocks
	std::vector<double> yref(static_cast<size_t>(dim), 0.0);
	for (size_t t = 0; t < plan.triples.size(); ++t) {
		const Triple&       tr = plan.triples[t];
		const BlockRef&     bl = plan.blocks[t];
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
	double yscale = 1e-300;
	for (double v : yref)
		yscale = std::max(yscale, std::fabs(v));
	const long long ops_n = plan.op_elems, bx_n = plan.bx_elems;
	if ((long long)pack.size() < ops_n)
		return fail("packed operators shorter than op_elems", (long long)pack.size(), ops_n);

	const int tiles[] = { 32, 64 }, bks[] = { 16, 32, 64 }, grids[] = { 7, 148, 296, 592 }, ipcs[] = { 1, 2, 4 };
	double    worst = 0.0;
	size_t    items = 0;
	for (int tile : tiles)
		for (int bk : bks)
			for (int grid : grids)
				for (int ipc : ipcs) {
					build_tile_lists(plan, tile, tile);
					build_persistent_schedule(plan, bk, grid, ipc);
					const std::string verdict = validate_persistent_schedule(plan, tile);
					if (!verdict.empty())
						return fail(("the validator rejects a good schedule: " + verdict).c_str());
					if (tile == 32 && bk == 16 && grid == 592 && ipc == 4) { // and rejects broken ones
						auto broken = [&](auto&& spoil) {
							KronPlan bad = plan;
							spoil(bad);
							return !validate_persistent_schedule(bad, tile).empty();
						};
						if (plan.n1_items > 0 && !broken([&](KronPlan& b) { b.items[0].c_off += 1; }))
							return fail("validator missed a moved pass-1 tile");
						if (plan.n1_items > 0
						    && !broken([&](KronPlan& b) { b.n1_of_j[size_t(b.items[0].producer)] += 1; }))
							return fail("validator missed a wrong pass-1 count");
						if (plan.items.size() > size_t(plan.n1_items)
						    && plan.items[size_t(plan.n1_items)].seg_end > plan.items[size_t(plan.n1_items)].seg_begin
						    && !broken([&](KronPlan& b) {
							       b.pseg2[size_t(b.items[size_t(b.n1_items)].seg_begin)].a_off += b.bx_elems;
						       }))
							return fail("validator missed a BX load out of range");
						for (size_t q = size_t(plan.n1_items); q < plan.items.size(); ++q)
							if (plan.items[q].kind == 2) {
								if (!broken([&](KronPlan& b) { b.items[q].part = (b.items[q].part + 1) % b.items[q].nsplit; }))
									return fail("validator missed a reused split slot");
								break;
							}
					}
					const auto& W = plan.items;
					items += W.size();
					const double nan = std::numeric_limits<double>::quiet_NaN();
					std::vector<double> bx(size_t(std::max<long long>(bx_n, 1)), nan), y(size_t(dim), nan);
					std::vector<int>    bxw(bx.size(), 0), yw(size_t(dim), 0);
					// pass 1
					std::vector<int> n1(size_t(np), 0);
					for (int q = 0; q < plan.n1_items; ++q) {
						const KronItem& w = W[size_t(q)];
						if (w.kind != 0 || w.seg_end - w.seg_begin != 1)
							return fail("pass-1 item", q, w.kind);
						const GemmSeg& g = plan.seg1[size_t(w.seg_begin)];
						if (w.producer != g.dep)
							return fail("pass-1 producer", q, w.producer);
						++n1[size_t(w.producer)];
						const long long j = w.producer, lo = plan.bx_off[size_t(j)],
						                hi = lo + plan.M[size_t(j)] * plan.l[size_t(j)];
						for (int n = w.n0; n < std::min(w.n0 + tile, w.N); ++n)
							for (int m = w.m0; m < std::min(w.m0 + tile, w.M); ++m) {
								double s = 0.0;
								for (int k = 0; k < g.K; ++k) {
									const long long ia = g.a_off + m + (long long)k * g.lda;
									const long long ib = g.b_off + k + (long long)n * g.ldb;
									if (ia < 0 || ia >= ops_n)
										return fail("pass-1 A load out of the operators", q, ia);
									if (ib < plan.xy_start[size_t(j)] || ib >= plan.xy_start[size_t(j) + 1])
										return fail("pass-1 x load out of X_j", q, ib);
									s += pack[size_t(ia)] * x[size_t(ib)];
								}
								const long long ic = w.c_off + m + (long long)n * w.ldc;
								if (ic < lo || ic >= hi)
									return fail("pass-1 store out of BX_j", q, ic);
								bx[size_t(ic)] = s;
								++bxw[size_t(ic)];
							}
					}
					for (int j = 0; j < np; ++j)
						if (n1[size_t(j)] != plan.n1_of_j[size_t(j)])
							return fail("n1_of_j", j, n1[size_t(j)]);
					for (size_t c = 0; c < bx.size() && bx_n > 0; ++c)
						if (bxw[c] > 1)
							return fail("BX element written twice", (long long)c, bxw[c]);
					// pass 2
					std::map<int, std::vector<const KronItem*>> split;
					std::map<long long, std::vector<double>>     slot;
					for (size_t q = size_t(plan.n1_items); q < W.size(); ++q) {
						const KronItem& w = W[q];
						if ((w.kind != 1 && w.kind != 2) || w.seg_end - w.seg_begin > kMaxItemSegs)
							return fail("pass-2 item", (long long)q, w.kind);
						if (w.seg_end > w.seg_begin) {
							const GemmSeg& s0 = plan.pseg2[size_t(w.seg_begin)];
							if (s0.a_off != w.seg0.a_off || s0.b_off != w.seg0.b_off || s0.K != w.seg0.K)
								return fail("seg0 copy", (long long)q, 0);
						}
						std::vector<double> part(size_t(tile) * size_t(tile), 0.0);
						for (int n = w.n0; n < std::min(w.n0 + tile, w.N); ++n)
							for (int m = w.m0; m < std::min(w.m0 + tile, w.M); ++m) {
								double s = 0.0;
								for (int e = w.seg_begin; e < w.seg_end; ++e) {
									const GemmSeg&  g  = plan.pseg2[size_t(e)];
									const long long lo = plan.bx_off[size_t(g.dep)],
									                hi = lo + plan.M[size_t(g.dep)] * plan.l[size_t(g.dep)];
									for (int k = 0; k < g.K; ++k) {
										const long long ia = g.a_off + m + (long long)k * g.lda;
										const long long ib = g.b_off + k + (long long)n * g.ldb;
										if (ia < lo || ia >= hi)
											return fail("pass-2 BX load outside its dependency", (long long)q, ia);
										if (bxw[size_t(ia)] != 1)
											return fail("pass-2 BX load of an element pass 1 did not write", (long long)q, ia);
										if (ib < 0 || ib >= ops_n)
											return fail("pass-2 A^T load out of the operators", (long long)q, ib);
										s += bx[size_t(ia)] * pack[size_t(ib)];
									}
								}
								if (w.kind == 1) {
									const long long ic = w.c_off + m + (long long)n * w.ldc;
									if (ic < 0 || ic >= dim)
										return fail("pass-2 store out of y", (long long)q, ic);
									y[size_t(ic)] = s;
									++yw[size_t(ic)];
								} else {
									part[size_t(m - w.m0) + size_t(n - w.n0) * size_t(tile)] = s;
								}
							}
						if (w.kind == 2) {
							if (w.part < 0 || w.part >= w.nsplit || w.slot + w.part >= plan.partial_slots)
								return fail("split part", (long long)q, w.part);
							if (!slot.emplace(w.slot + w.part, part).second)
								return fail("split slot used twice", w.slot + w.part, 0);
							split[w.tile].push_back(&w);
						}
					}
					if ((int)split.size() != plan.n_split_tiles)
						return fail("split tiles", (long long)split.size(), plan.n_split_tiles);
					for (const auto& kv : split) {
						const auto& parts = kv.second;
						const KronItem& w0 = *parts[0];
						if ((int)parts.size() != w0.nsplit)
							return fail("parts of a split tile", kv.first, (long long)parts.size());
						for (const KronItem* p : parts)
							if (p->c_off != w0.c_off || p->m0 != w0.m0 || p->n0 != w0.n0 || p->slot != w0.slot)
								return fail("parts disagree on their tile", kv.first, 0);
						for (int n = w0.n0; n < std::min(w0.n0 + tile, w0.N); ++n)
							for (int m = w0.m0; m < std::min(w0.m0 + tile, w0.M); ++m) {
								double s = 0.0;
								for (int p = 0; p < w0.nsplit; ++p) // the last part sums the slots in order
									s += slot[w0.slot + p][size_t(m - w0.m0) + size_t(n - w0.n0) * size_t(tile)];
								const long long ic = w0.c_off + m + (long long)n * w0.ldc;
								if (ic < 0 || ic >= dim)
									return fail("split store out of y", kv.first, ic);
								y[size_t(ic)] = s;
								++yw[size_t(ic)];
							}
					}
					for (long long e = 0; e < dim; ++e) {
						if (yw[size_t(e)] != 1)
							return fail("y element not written exactly once", e, yw[size_t(e)]);
						worst = std::max(worst, std::fabs(y[size_t(e)] - yref[size_t(e)]) / yscale);
					}
				}
	if (!(worst <= 1e-12))
		return fail("result differs from H*x", (long long)(worst * 1e15), 0);
	std::printf("ok %.3e %zu\n", worst, items);
	return 0;
}
