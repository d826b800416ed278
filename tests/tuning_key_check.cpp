// CPU check of the autotuner's cache key (tuning_key in kron_plan.cpp): a
// sector keeps its key when a few patches change by a state or two (as
// between consecutive sweep steps), and gets another key for another shape,
// term count or GPU.  Sectors are spin-chain-like: patch p has l = r = n_p
// states (a discretised Gaussian of np groups), three terms couple p with
// itself and two couple p with p - 1 and p + 1.
#include "kron_plan.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

using namespace dmrgpp;

namespace {

std::vector<size_t> gaussian(size_t total, int np, double sigma)
{
	std::vector<double> w(static_cast<size_t>(np));
	double              sum = 0.0;
	for (int p = 0; p < np; ++p) {
		const double x = p - (np - 1) / 2.0;
		w[size_t(p)]   = std::exp(-x * x / (2 * sigma * sigma));
		sum += w[size_t(p)];
	}
	std::vector<size_t> n(static_cast<size_t>(np));
	size_t              used = 0;
	for (int p = 0; p < np; ++p) {
		n[size_t(p)] = std::max<size_t>(1, size_t(double(total) * w[size_t(p)] / sum));
		used += n[size_t(p)];
	}
	n[size_t(np / 2)] += total > used ? total - used : 0;
	return n;
}

std::string key(const std::vector<size_t>& n, int nop, const char* gpu)
{
	const size_t np = n.size();
	const size_t nt = np * np * size_t(nop);
	std::vector<std::vector<double>> store;
	std::vector<const double*>       A(nt, nullptr), B(nt, nullptr);
	std::vector<size_t>              ldA(nt, 0), ldB(nt, 0);
	store.reserve(2 * nt);
	for (int k = 0; k < nop; ++k)
		for (size_t i = 0; i < np; ++i)
			for (size_t j = 0; j < np; ++j) {
				const bool diag = k < 3 && i == j;
				const bool hop  = k >= 3 && (k == 3 ? j + 1 == i : i + 1 == j);
				if (!diag && !hop)
					continue;
				const size_t ix = i + j * np + size_t(k) * np * np;
				store.emplace_back(n[i] * n[j], 1.0);
				A[ix]   = store.back().data();
				ldA[ix] = n[i];
				store.emplace_back(n[i] * n[j], 1.0);
				B[ix]   = store.back().data();
				ldB[ix] = n[i];
			}
	KronPlan          plan;
	const std::string msg = build_kron_plan(size_t(nop), np, n.data(), n.data(), A.data(), ldA.data(), B.data(),
	                                        ldB.data(), 64, 64, plan, nullptr);
	if (!msg.empty()) {
		std::printf("FAIL plan %s\n", msg.c_str());
		std::exit(1);
	}
	return tuning_key(plan, gpu);
}

} // namespace

int main()
{
	const char* gpu = "NVIDIA B200";
	const auto  n   = gaussian(1024, 21, 4.0);
	const auto  k0  = key(n, 5, gpu);
	int         bad = 0;
	auto expect = [&](bool ok, const char* what) {
		if (!ok) {
			std::printf("FAIL %s\n", what);
			++bad;
		}
	};
	expect(key(n, 5, gpu) == k0, "same sector, same key");
	// a sweep step: a few patches gain or lose a state or two
	auto m = n;
	m[10] += 2;
	m[9] -= 1;
	m[12] += 1;
	m[4] -= 1;
	expect(key(m, 5, gpu) == k0, "patches changed by a state or two keep the key");
	expect(key(gaussian(4096, 21, 4.0), 5, gpu) != k0, "a four times larger sector gets another key");
	expect(key(n, 4, gpu) != k0, "another number of terms gets another key");
	expect(key(n, 5, "another GPU") != k0, "another GPU gets another key");
	if (bad)
		return 1;
	std::printf("ok %s\n", k0.c_str());
	return 0;
}
