// Host emulation of the TF32x3 tensor-core passes over the chunked,
// pre-swizzled operand layout that build_mixed_plan produces.  Checks, on
// the CPU, what the kernel in tc_gemm.cu relies on:
//   * every operand buffer is a whole number of 128-byte rows (a 2-D TMA
//     tensor); every tiled TMA load the producer would issue (A and B tiles
//     of every k-chunk of every segment) starts inside its buffer at an int
//     row, and the valid output rows and columns read rows of one chunk of
//     their own matrix (rows past the buffer arrive as zeros, as the TMA unit
//     fills them);
//   * the per-CTA tile runs (balance_tiles) are a permutation of the tiles;
//   * K-split pass-2 tiles: slots in range, every part present, the parts'
//     sums are the tile's output;
//   * the device-side operator packing (mixed_pack_jobs) reproduces the host
//     packing bit for bit;
//   * the staged FP64 upload (build_upload_plan, fill_upload_chunk and the
//     placement of upload_place_kernel) writes every packed position once,
//     with the host packing's value, also for blocks whose leading dimension
//     exceeds their rows;
//   * the epilogue's stores stay inside their buffers;
//   * pass 1 + pass 2 computed from these buffers (hi*hi + hi*lo + lo*hi in
//     double) reproduce the FP64 H*x;
//   * validate_mixed_plan (the library's debug-mode check) accepts the plan
//     and rejects spoilt copies.
// Usage: mixed_layout_check seed npatches noperator max_size bn
// Prints "ok <max relative error>" or "FAIL <reason>" (exit code 1).
#include "kron_plan.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <map>
#include <set>
#include <random>
#include <tuple>
#include <vector>

using namespace dmrgpp;

namespace {

int fail(const char* why, long long a = 0, long long b = 0)
{
	std::printf("FAIL %s %lld %lld\n", why, a, b);
	return 1;
}

struct Buf {
	const float* hi;
	const float* lo;
	long long    n;
};

} // namespace

int main(int argc, char** argv)
{
	if (argc < 6)
		return fail("usage");
	const unsigned seed = unsigned(std::atoi(argv[1]));
	const int      np   = std::atoi(argv[2]);
	const int      nop  = std::atoi(argv[3]);
	const int      maxs = std::atoi(argv[4]);
	const int      bn   = std::atoi(argv[5]);
	std::mt19937_64 rng(seed);
	std::uniform_int_distribution<int>     size(1, maxs);
	std::uniform_real_distribution<double> val(-1.0, 1.0);
	std::uniform_real_distribution<double> coin(0.0, 1.0);

	std::vector<size_t> l(np), r(np);
	for (int p = 0; p < np; ++p) {
		l[p] = size_t(size(rng));
		r[p] = size_t(size(rng));
	}
	const size_t               nt = size_t(np) * np * nop;
	std::vector<std::vector<double>> Ast(nt), Bst(nt);
	std::vector<const double*> A(nt, nullptr), B(nt, nullptr);
	std::vector<size_t>        ldA(nt, 0), ldB(nt, 0);
	for (int k = 0; k < nop; ++k)
		for (int j = 0; j < np; ++j)
			for (int i = 0; i < np; ++i) {
				if (coin(rng) < 0.35)
					continue;
				const size_t ix = size_t(i) + size_t(j) * np + size_t(k) * np * np;
				// some blocks sit in larger arrays (leading dimension > rows)
				ldA[ix] = l[i] + (coin(rng) < 0.3 ? 3 : 0);
				ldB[ix] = r[i] + (coin(rng) < 0.3 ? 5 : 0);
				Ast[ix].resize(ldA[ix] * l[j]);
				Bst[ix].resize(ldB[ix] * r[j]);
				for (double& v : Ast[ix])
					v = val(rng);
				for (double& v : Bst[ix])
					v = val(rng);
				A[ix]   = Ast[ix].data();
				B[ix]   = Bst[ix].data();
			}

	KronPlan            plan;
	std::string         msg;
	std::vector<float>  ohi, olo;
	std::vector<int>    xmap;
	PackBuffer          pack64;
	msg = build_kron_plan(size_t(nop), size_t(np), l.data(), r.data(), A.data(), ldA.data(),
	                      B.data(), ldB.data(), 64, 64, plan, &pack64);
	if (!msg.empty())
		return fail(msg.c_str());
	msg = build_mixed_plan(plan, bn, &ohi, &olo, &xmap);
	if (!msg.empty())
		return fail(msg.c_str());
	// the library's debug-mode check accepts the plan and rejects spoilt copies
	msg = validate_mixed_plan(plan);
	if (!msg.empty())
		return fail(("the validator rejects a good plan: " + msg).c_str());
	if (!plan.mixed.seg2.empty()) {
		KronPlan bad = plan;
		bad.mixed.seg2.back().a_off += bad.mixed.bxs_elems / 32;
		if (validate_mixed_plan(bad).empty())
			return fail("validator missed a load outside its buffer");
	}
	if (!plan.mixed.tile2.empty()) {
		KronPlan bad = plan;
		bad.mixed.tile2.back().c_off += plan.dim();
		if (validate_mixed_plan(bad).empty())
			return fail("validator missed a y store out of bounds");
	}
	// per-CTA runs (balance_tiles): a permutation of the tiles, runs cover all
	for (int pass_no = 0; pass_no < 2; ++pass_no) {
		std::vector<GemmTile>&       tl   = pass_no ? plan.mixed.tile2 : plan.mixed.tile1;
		const std::vector<GemmSeg>&  sg   = pass_no ? plan.mixed.seg2 : plan.mixed.seg1;
		auto key = [](const GemmTile& t) { return std::make_tuple(t.c_off, t.m0, t.n0, t.seg_begin); };
		std::vector<std::tuple<long long, int, int, int>> before, after;
		for (const GemmTile& t : tl)
			before.push_back(key(t));
		std::vector<int> starts;
		const int        G = balance_tiles(tl, sg, 7, starts);
		if (G != std::min<int>(7, int(tl.size())) || int(starts.size()) != std::max(G, 1) + 1
		    || starts.front() != 0 || starts.back() != int(tl.size()))
			return fail("tile runs do not cover the tiles", G, long(starts.size()));
		for (size_t b = 0; b + 1 < starts.size(); ++b)
			if (starts[b] > starts[b + 1])
				return fail("tile runs not ordered", long(b), 0);
		for (const GemmTile& t : tl)
			after.push_back(key(t));
		std::sort(before.begin(), before.end());
		std::sort(after.begin(), after.end());
		if (before != after)
			return fail("tile runs are not a permutation", pass_no, 0);
	}
	// the staged upload (build_upload_plan + fill_upload_chunk on the host,
	// the placement of upload_place_kernel emulated here) writes exactly the
	// packed FP64 operators: every position once, with the host packing's value
	{
		// chunks smaller than the longest column (seeds 1-3) take the
		// longest column as their size
		const long long chunk = (seed % 4 == 1 ? 20 : 700) + 37 * (long long)(seed % 11);
		const long long job   = 150 + 13 * (long long)(seed % 7);
		const UploadPlan up   = build_upload_plan(plan, chunk, job);
		long long        longest = 1;
		for (const Triple& tr : plan.triples)
			longest = std::max({ longest, plan.r[tr.i], plan.l[tr.i] });
		if (up.chunk_elems != std::max(chunk, longest))
			return fail("upload chunk size", up.chunk_elems, std::max(chunk, longest));
		std::vector<double> out(pack64.size(), std::numeric_limits<double>::quiet_NaN());
		std::vector<char>   hit(pack64.size(), 0);
		long long           written = 0, expect = 0;
		for (size_t t = 0; t < plan.triples.size(); ++t) {
			const Triple& tr = plan.triples[t];
			expect += plan.r[tr.i] * plan.r[tr.j] + plan.l[tr.i] * plan.l[tr.j];
		}
		if (up.chunk_begin.size() != up.chunks() + 1 || up.chunk_begin.back() != up.jobs.size())
			return fail("upload chunks do not cover the jobs", long(up.chunks()), long(up.jobs.size()));
		for (size_t c = 0; c < up.chunks(); ++c) {
			if (up.chunk_fill[c] > up.chunk_elems)
				return fail("upload chunk overfilled", up.chunk_fill[c], up.chunk_elems);
			std::vector<double> buf(size_t(up.chunk_elems), 0.0);
			const size_t        n = up.chunk_begin[c + 1] - up.chunk_begin[c];
			fill_upload_chunk(up, c, 0, n / 2, buf.data()); // two calls, as two threads would
			fill_upload_chunk(up, c, n / 2, n, buf.data());
			for (size_t q = up.chunk_begin[c]; q < up.chunk_begin[c + 1]; ++q) {
				const UploadJob& j = up.jobs[q];
				if (j.src < 0 || j.src + (long long)j.rows * j.cols > up.chunk_fill[c])
					return fail("upload part outside its chunk", j.src, up.chunk_fill[c]);
				if ((long long)j.rows * j.cols > std::max<long long>(job, j.rows))
					return fail("upload part too large", j.rows, j.cols);
				for (int cc = 0; cc < j.cols; ++cc)
					for (int qq = 0; qq < j.rows; ++qq) {
						const long long d = j.transpose ? j.dst + cc + (long long)qq * j.ld_dst
						                                : j.dst + qq + (long long)cc * j.ld_dst;
						if (d < 0 || d >= (long long)out.size())
							return fail("upload placement out of bounds", d, (long long)out.size());
						if (hit[size_t(d)]++)
							return fail("upload writes a position twice", d, 0);
						out[size_t(d)] = buf[size_t(j.src + qq + (long long)cc * j.rows)];
						++written;
					}
			}
		}
		if (written != expect)
			return fail("upload writes the wrong number of elements", written, expect);
		for (size_t e = 0; e < out.size(); ++e)
			if (hit[e] && out[e] != pack64[e])
				return fail("upload differs from the host packing", (long long)e, 0);
	}
	const MixedPlan& mp = plan.mixed;
	const long long  D  = plan.dim();
	// the device packing (mixed_pack_jobs over the FP64 packed operators,
	// the arithmetic of pack_tf32_kernel) gives exactly the host packing
	{
		std::vector<float> dhi(size_t(mp.ops_elems), 0.f), dlo(size_t(mp.ops_elems), 0.f);
		for (const PackJob& jb : mixed_pack_jobs(plan))
			for (long long e = 0; e < (long long)jb.rows * jb.cols; ++e) {
				const long long q = e % jb.rows, c = e / jb.rows;
				const long long row = jb.swap ? c : jb.row0 + q, k = jb.swap ? q : c;
				const long long d = jb.dst + chunked_offset(jb.dst_rows, row, k);
				const long long sidx = jb.src + q + c * (long long)jb.ld;
				if (d < 0 || d >= mp.ops_elems || sidx < 0 || sidx >= (long long)pack64.size())
					return fail("pack job out of bounds", d, sidx);
				split_tf32(pack64[size_t(sidx)], &dhi[size_t(d)], &dlo[size_t(d)]);
			}
		if (dhi != ohi || dlo != olo)
			return fail("device-style packing differs from the host packing");
	}

	std::vector<double> x(static_cast<size_t>(D)), y_ref(static_cast<size_t>(D), 0.0);
	for (double& v : x)
		v = val(rng);
	// FP64 reference: Y_i = sum B_k(i,j) X_j A_k(i,j)^T
	for (const Triple& t : plan.triples) {
		const size_t ix = size_t(t.i) + size_t(t.j) * np + size_t(t.k) * np * np;
		const long long ri = r[t.i], rj = r[t.j], li = l[t.i], lj = l[t.j];
		for (long long a = 0; a < ri; ++a)
			for (long long b = 0; b < li; ++b) {
				double s = 0;
				for (long long c = 0; c < rj; ++c)
					for (long long d = 0; d < lj; ++d)
						s += B[ix][a + c * (long long)ldB[ix]] * x[size_t(plan.xy_start[t.j] + c + d * rj)]
						    * A[ix][b + d * (long long)ldA[ix]];
				y_ref[size_t(plan.xy_start[t.i] + a + b * ri)] += s;
			}
	}

	// x split (zero K padding, like the cleared device buffer + split_x)
	std::vector<float> xs_hi(size_t(mp.xs_elems), 0.f), xs_lo(size_t(mp.xs_elems), 0.f);
	for (long long e = 0; e < D; ++e) {
		const int d = xmap[size_t(e)];
		if (d < 0 || d >= mp.xs_elems)
			return fail("x map out of range", e, d);
		split_tf32(x[size_t(e)], &xs_hi[size_t(d)], &xs_lo[size_t(d)]);
	}
	const float nanf = std::numeric_limits<float>::quiet_NaN();
	std::vector<float>  bx_hi(size_t(mp.bxs_elems), nanf), bx_lo(size_t(mp.bxs_elems), nanf);
	std::vector<double> y(size_t(D), std::numeric_limits<double>::quiet_NaN());

	const int BM = mp.bm;
	std::map<long long, double>      split_sum;
	std::map<int, std::set<int>>     split_parts;
	std::map<int, int>               split_n;
	// emulate one pass: every operand buffer is a 2-D TMA tensor
	// [row][32 floats]; a load of `box` rows from buffer row y reads rows
	// y .. y + box - 1 (zeros past the buffer's end).  Returns 0 on success.
	auto pass = [&](const std::vector<GemmSeg>& segs, const std::vector<GemmTile>& tiles, Buf Ab,
	                Buf Bb, bool pass1) -> int {
		if (Ab.n % 32 != 0 || Bb.n % 32 != 0)
			return fail("buffer not a whole number of rows", Ab.n, Bb.n);
		const long long arows = Ab.n / 32, brows = Bb.n / 32;
		std::vector<double> acc(size_t(BM) * bn);
		for (const GemmTile& t : tiles) {
			std::fill(acc.begin(), acc.end(), 0.0);
			int chunks = 0;
			for (int s = t.seg_begin; s < t.seg_end; ++s) {
				const GemmSeg& g = segs[size_t(s)];
				if (g.K % 32 != 0 || g.lda <= 0 || g.ldb <= 0 || g.lda % 8 != 0 || g.ldb % 8 != 0)
					return fail("segment fields", g.K, g.lda);
				// the tile's valid rows stay inside one chunk of its matrix
				if (t.m0 + std::min(BM, t.M - t.m0) > g.lda || t.n0 + std::min(bn, t.N - t.n0) > g.ldb)
					return fail("valid rows past the matrix", g.lda, g.ldb);
				for (int c = 0; c < g.K / 32; ++c, ++chunks) {
					const long long ya = g.a_off + t.m0 + (long long)c * g.lda;
					const long long yb = g.b_off + t.n0 + (long long)c * g.ldb;
					if (ya < 0 || yb < 0 || ya > INT_MAX || yb > INT_MAX || ya >= arows || yb >= brows)
						return fail("tile row outside its buffer", ya, yb);
					auto val = [&](const Buf& b, long long nrows, long long row, int k, bool hi) -> double {
						if (row >= nrows)
							return 0.0; // TMA out-of-bounds fill
						return hi ? b.hi[row * 32 + k] : b.lo[row * 32 + k];
					};
					for (int m = 0; m < BM; ++m)
						for (int n = 0; n < bn; ++n) {
							double sum = 0;
							for (int k = 0; k < 32; ++k) {
								const double ah = val(Ab, arows, ya + m, k, true), al = val(Ab, arows, ya + m, k, false);
								const double bh = val(Bb, brows, yb + n, k, true), bl = val(Bb, brows, yb + n, k, false);
								sum += ah * bh + ah * bl + al * bh;
							}
							acc[size_t(m) * bn + n] += sum;
						}
				}
			}
			if (pass1 && t.c_off % 32 != 0)
				return fail("BX matrix not on a 32-float row", t.c_off, 0);
			// pass 1's staged stores: a warp's 32 rows (all inside the matrix)
			// of one chunk as one 32-row box at buffer row R, which must be
			// the rows the per-element offsets below name
			for (int q = 0; pass1 && q < 4; ++q) {
				if (t.m0 + 32 * q + 32 > t.M)
					continue;
				for (int c0 = 0; c0 < bn && t.n0 + c0 < t.N; c0 += 32) {
					const int       col0 = t.n0 + c0;
					const long long R    = t.c_off / 32 + (long long)(col0 >> 5) * t.ldc + t.m0 + 32 * q;
					const long long o0   = t.c_off + (long long)(col0 >> 5) * t.ldc * 32
					    + (long long)(t.m0 + 32 * q) * 32;
					if (R < 0 || R > INT_MAX || (R + 32) * 32 > mp.bxs_elems || R * 32 != o0)
						return fail("staged BX store rows", R, mp.bxs_elems);
				}
			}
			for (int m = 0; m < BM; ++m) {
				const int grow = t.m0 + m;
				for (int c0 = 0; c0 < bn; c0 += 32) {
					const int col0 = t.n0 + c0;
					if (grow >= t.M || col0 >= t.N)
						continue;
					for (int e = 0; e < 32; ++e) {
						const int    gcol = col0 + e;
						const double v    = chunks ? acc[size_t(m) * bn + c0 + e] : 0.0;
						if (pass1) {
							const long long o = t.c_off + (long long)(col0 >> 5) * t.ldc * 32
							    + (long long)grow * 32 + e;
							if (o < 0 || o >= mp.bxs_elems)
								return fail("BX store out of bounds", o, mp.bxs_elems);
							float h, lo;
							split_tf32(gcol < t.N ? double(float(v)) : 0.0, &h, &lo);
							bx_hi[size_t(o)] = h;
							bx_lo[size_t(o)] = lo;
						} else if (gcol < t.N) {
							const long long o = t.c_off + (long long)gcol * t.ldc + grow;
							if (o < 0 || o >= D)
								return fail("y store out of bounds", o, D);
							if (t.nsplit >= 2) { // part of a K-split tile: slot, summed later
								if (t.slot < 0 || t.split_part < 0 || t.split_part >= t.nsplit
								    || t.slot + t.nsplit > mp.split_slots)
									return fail("split slot out of range", t.slot, t.split_part);
								split_sum[o] = (split_sum.count(o) ? split_sum[o] : 0.0) + double(float(v));
								split_parts[t.split_tile].insert(t.split_part);
								split_n[t.split_tile] = t.nsplit;
							} else {
								y[size_t(o)] = v;
							}
						}
					}
				}
			}
		}
		return 0;
	};
	const Buf ops {ohi.data(), olo.data(), mp.ops_elems};
	const Buf xsb {xs_hi.data(), xs_lo.data(), mp.xs_elems};
	const Buf bxb {bx_hi.data(), bx_lo.data(), mp.bxs_elems};
	if (pass(mp.seg1, mp.tile1, ops, xsb, true))
		return 1;
	if (pass(mp.seg2, mp.tile2, bxb, ops, false))
		return 1;
	// every split tile got all of its parts, and their sums are its output
	if (int(split_parts.size()) != mp.n_split_tiles)
		return fail("split tiles without parts", long(split_parts.size()), mp.n_split_tiles);
	for (const auto& kv : split_parts)
		if (int(kv.second.size()) != split_n[kv.first])
			return fail("split tile missing parts", kv.first, long(kv.second.size()));
	for (const auto& kv : split_sum)
		y[size_t(kv.first)] = kv.second;
	double err = 0, ref = 0;
	for (long long e = 0; e < D; ++e) {
		if (!std::isfinite(y[size_t(e)]))
			return fail("y not written or not finite", e, 0);
		err = std::max(err, std::fabs(y[size_t(e)] - y_ref[size_t(e)]));
		ref = std::max(ref, std::fabs(y_ref[size_t(e)]));
	}
	const double rel = ref > 0 ? err / ref : err;
	if (rel > 1e-5)
		return fail("result differs from FP64", (long long)(rel * 1e9), 0);
	std::printf("ok %.3e split_tiles %d\n", rel, mp.n_split_tiles);
	return 0;
}
