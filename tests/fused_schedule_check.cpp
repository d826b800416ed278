// Host emulation of the fused H*x launch (kron_fused.cu) over the schedule
// that build_fused_schedule produces.  Checks, on the CPU, what the kernel
// relies on:
//   * the item list is whole clusters; in every cluster the parts of a tile
//     sit at ranks rank0 .. rank0 + nparts - 1 and agree on the tile; empty
//     slots have nparts = 0;
//   * every output tile of every patch appears once, its parts cover its
//     units in order, and every unit of the patch's contributing triples
//     (times every unit-wide chunk of X_j's columns) appears once;
//   * every operand element the kernel loads (with its zero-fill predicates)
//     lies inside its block of the packed operators or of x, and every store
//     inside Y_i;
//   * the per-part products summed in part order (the cluster reduction)
//     reproduce H*x computed directly from the caller's blocks;
//   * validate_fused_schedule (the library's debug-mode check) accepts every
//     schedule and rejects spoilt copies.
// Usage: fused_schedule_check seed npatches noperator max_size
// Prints "ok <max relative error> <items>" or "FAIL <reason>" (exit code 1).
#include "kron_plan.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <random>
#include <set>
#include <tuple>
#include <vector>

using namespace dmrgpp;

namespace {

int fail(const char* why, long long a = 0, long long b = 0)
{
	std::printf("FAIL %s %lld %lld\n", why, a, b);
	return 1;
}

struct Shape {
	int bm, cw, bn, cluster, parts_per_sm, sms;
};

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

	std::vector<size_t> l(np), r(np);
	for (int p = 0; p < np; ++p) {
		l[p] = size_t(size(rng));
		r[p] = size_t(size(rng));
	}
	const size_t                     nt = size_t(np) * np * nop;
	std::vector<std::vector<double>> Ast(nt), Bst(nt);
	std::vector<const double*>       A(nt, nullptr), B(nt, nullptr);
	std::vector<size_t>              ldA(nt, 0), ldB(nt, 0);
	for (int k = 0; k < nop; ++k)
		for (int j = 0; j < np; ++j)
			for (int i = 0; i < np; ++i) {
				if (coin(rng) < 0.4)
					continue;
				const size_t ix = size_t(i) + size_t(j) * np + size_t(k) * np * np;
				ldA[ix]         = l[i] + (coin(rng) < 0.3 ? 2 : 0);
				ldB[ix]         = r[i] + (coin(rng) < 0.3 ? 3 : 0);
				Ast[ix].resize(ldA[ix] * l[j]);
				Bst[ix].resize(ldB[ix] * r[j]);
				for (double& v : Ast[ix])
					v = val(rng);
				for (double& v : Bst[ix])
					v = val(rng);
				A[ix] = Ast[ix].data();
				B[ix] = Bst[ix].data();
			}
	KronPlan   plan;
	PackBuffer pack;
	std::string msg = build_kron_plan(size_t(nop), size_t(np), l.data(), r.data(), A.data(), ldA.data(),
	                                  B.data(), ldB.data(), 32, 32, plan, &pack);
	if (!msg.empty())
		return fail(msg.c_str());
	const long long dim = plan.dim();
	std::vector<double> x(static_cast<size_t>(dim));
	for (double& v : x)
		v = val(rng);
	// direct H*x from the caller's blocks
	std::vector<double> yref(size_t(dim), 0.0);
	for (size_t t = 0; t < plan.triples.size(); ++t) {
		const Triple&   tr = plan.triples[t];
		const BlockRef& bl = plan.blocks[t];
		const long long ri = plan.r[tr.i], li = plan.l[tr.i], rj = plan.r[tr.j], lj = plan.l[tr.j];
		const double*   X  = x.data() + plan.xy_start[tr.j];
		double*         Y  = yref.data() + plan.xy_start[tr.i];
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
	double    yscale = 1e-300;
	for (double v : yref)
		yscale = std::max(yscale, std::fabs(v));

	const Shape shapes[] = { { 16, 128, 128, 8, 2, 148 }, { 32, 64, 128, 8, 1, 148 },
		                     { 32, 128, 128, 8, 4, 148 }, { 16, 64, 64, 16, 2, 148 },
		                     { 32, 32, 128, 16, 4, 7 },   { 16, 64, 64, 8, 1, 3 } };
	double      worst = 0.0;
	size_t      items = 0;
	for (const Shape& s : shapes) {
		build_fused_schedule(plan, s.bm, s.bn, s.cw, s.cluster, s.parts_per_sm, s.sms);
		const std::string verdict = validate_fused_schedule(plan, s.bm, s.bn, s.cluster);
		if (!verdict.empty())
			return fail(("the validator rejects a good schedule: " + verdict).c_str());
		if (!plan.funits.empty()) { // and rejects spoilt copies
			KronPlan bad = plan;
			bad.funits.back().x_off += dim;
			if (validate_fused_schedule(bad, s.bm, s.bn, s.cluster).empty())
				return fail("validator missed an x load out of range");
			bad = plan;
			bad.funits.front().at_off += plan.op_elems;
			if (validate_fused_schedule(bad, s.bm, s.bn, s.cluster).empty())
				return fail("validator missed an A^T load out of range");
		}
		const auto& I = plan.fitems;
		const auto& U = plan.funits;
		items += I.size();
		if (I.size() % size_t(s.cluster) != 0)
			return fail("items not whole clusters", long(I.size()), s.cluster);
		// clusters: parts contiguous, one tile per run of parts
		std::map<std::tuple<int, int, int>, std::vector<int>> tile_items; // (patch off, m0, n0)
		for (size_t c = 0; c < I.size(); c += size_t(s.cluster)) {
			for (int rk = 0; rk < s.cluster; ++rk) {
				const FusedItem& it = I[c + size_t(rk)];
				if (it.nparts == 0)
					continue;
				if (it.nparts > s.cluster || it.part < 0 || it.part >= it.nparts || it.rank0 + it.part != rk
				    || it.rank0 + it.nparts > s.cluster)
					return fail("part placement", long(c), rk);
				const FusedItem& p0 = I[c + size_t(it.rank0)];
				if (p0.y_off != it.y_off || p0.m0 != it.m0 || p0.n0 != it.n0 || p0.nparts != it.nparts)
					return fail("parts of one tile disagree", long(c), rk);
				if (it.part > 0 && I[c + size_t(rk) - 1].u_end != it.u_begin)
					return fail("parts not contiguous in units", long(c), rk);
				tile_items[{ int(it.y_off), it.m0, it.n0 }].push_back(int(c) + rk);
			}
		}
		// every tile of every patch once; units cover the contributions once
		std::vector<double> y(size_t(dim), std::nan(""));
		size_t              tiles = 0;
		for (int i = 0; i < np; ++i) {
			const long long M = plan.r[size_t(i)], N = plan.l[size_t(i)];
			std::vector<std::tuple<long long, long long>> expect; // (triple, c0) in order
			for (size_t t = 0; t < plan.triples.size(); ++t)
				if (plan.triples[t].i == i)
					for (long long c0 = 0; c0 < plan.l[size_t(plan.triples[t].j)]; c0 += s.cw)
						expect.emplace_back((long long)t, c0);
			for (long long m0 = 0; m0 < M; m0 += s.bm)
				for (long long n0 = 0; n0 < N; n0 += s.bn) {
					++tiles;
					auto f = tile_items.find({ int(plan.xy_start[size_t(i)]), int(m0), int(n0) });
					if (f == tile_items.end())
						return fail("tile missing", i, m0);
					const std::vector<int>& parts = f->second;
					const FusedItem&        first = I[size_t(parts.front())];
					if (int(parts.size()) != first.nparts || first.M != M || first.N != N)
						return fail("tile parts", i, long(parts.size()));
					if (size_t(I[size_t(parts.back())].u_end - first.u_begin) != expect.size())
						return fail("tile units", i, long(expect.size()));
					const long long Mt = std::min<long long>(s.bm, M - m0), Nt = std::min<long long>(s.bn, N - n0);
					std::vector<std::vector<double>> partial;
					for (int q : parts) {
						const FusedItem& it = I[size_t(q)];
						std::vector<double> acc(size_t(s.bm * s.bn), 0.0);
						for (int u = it.u_begin; u < it.u_end; ++u) {
							const FusedUnit& d  = U[size_t(u)];
							const auto&      ex = expect[size_t(u - first.u_begin)];
							const Triple&    tr = plan.triples[size_t(std::get<0>(ex))];
							const long long  c0 = std::get<1>(ex);
							if (d.rj != plan.r[size_t(tr.j)] || d.lj != plan.l[size_t(tr.j)] || d.ldb != plan.M[size_t(tr.j)]
							    || d.cw != int(std::min<long long>(s.cw, d.lj - c0)))
								return fail("unit fields", i, u);
							// loads of the first product (valid ones only: the rest are zero fill)
							std::vector<double> T(size_t(s.bm * s.cw), 0.0);
							for (int kk = 0; kk < d.rj; ++kk)
								for (long long m = 0; m < Mt; ++m) {
									const long long ab = d.b_off + (long long)kk * d.ldb + m0 + m;
									const long long lo = plan.bstack_off[size_t(tr.j)] + plan.row_off[size_t(std::get<0>(ex))];
									if (ab < lo || ab >= plan.bstack_off[size_t(tr.j)] + plan.M[size_t(tr.j)] * plan.r[size_t(tr.j)]
									    || (ab - plan.bstack_off[size_t(tr.j)]) % d.ldb - plan.row_off[size_t(std::get<0>(ex))] >= M)
										return fail("B operand out of its block", i, u);
									for (int n = 0; n < d.cw; ++n) {
										const long long xb = d.x_off + (long long)n * d.rj + kk;
										if (xb < plan.xy_start[size_t(tr.j)] || xb >= plan.xy_start[size_t(tr.j) + 1])
											return fail("x operand out of X_j", i, u);
										T[size_t(m * s.cw + n)] += pack[size_t(ab)] * x[size_t(xb)];
									}
								}
							for (int kk = 0; kk < d.cw; ++kk)
								for (long long n = 0; n < Nt; ++n) {
									const long long ab = d.at_off + (n0 + n) * d.lj + kk;
									if (ab < plan.at_off[size_t(std::get<0>(ex))]
									    || ab >= plan.at_off[size_t(std::get<0>(ex))] + plan.l[size_t(tr.j)] * N)
										return fail("A^T operand out of its block", i, u);
									for (long long m = 0; m < Mt; ++m)
										acc[size_t(n * s.bm + m)] += T[size_t(m * s.cw + kk)] * pack[size_t(ab)];
								}
						}
						partial.push_back(std::move(acc));
					}
					// the cluster reduction: slice p of the tile by part p, parts summed in order
					const long long E = Mt * Nt;
					for (size_t p = 0; p < parts.size(); ++p) {
						const long long e0 = E * (long long)p / (long long)parts.size();
						const long long e1 = E * (long long)(p + 1) / (long long)parts.size();
						for (long long e = e0; e < e1; ++e) {
							const long long col = e / Mt, row = e % Mt;
							double          sum = partial[0][size_t(col * s.bm + row)];
							for (size_t q = 1; q < parts.size(); ++q)
								sum += partial[q][size_t(col * s.bm + row)];
							const long long yo = plan.xy_start[size_t(i)] + (n0 + col) * M + m0 + row;
							if (yo < plan.xy_start[size_t(i)] || yo >= plan.xy_start[size_t(i) + 1])
								return fail("store out of Y_i", i, e);
							if (!std::isnan(y[size_t(yo)]))
								return fail("element stored twice", i, e);
							y[size_t(yo)] = sum;
						}
					}
				}
		}
		if (tiles != tile_items.size())
			return fail("extra tiles", long(tiles), long(tile_items.size()));
		for (long long e = 0; e < dim; ++e) {
			if (std::isnan(y[size_t(e)]))
				return fail("element never stored", e, 0);
			worst = std::max(worst, std::fabs(y[size_t(e)] - yref[size_t(e)]) / yscale);
		}
	}
	if (!(worst < 1e-13))
		return fail("result differs", long(worst * 1e16), 0);
	std::printf("ok %.3e %zu\n", worst, items);
	return 0;
}
