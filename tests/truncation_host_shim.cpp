// A C entry to the host part of dmrgpp_density_truncate (tridiag.cpp), built
// by tests/test_truncation_host.py with g++: the eigenvalue phase
// (group_eigenvalues) and the kept eigenvectors (group_eigenvectors, then
// V = Q Z by apply_q, the host form of the device's back-transformation), so
// that the pipeline can be checked against the numpy oracle on the CPU.
#include "tridiag.h"

#include <cstddef>
#include <vector>

namespace {
std::vector<dmrgpp::GroupReduction> g_red; // the reductions of the last shim_eigenvalues
}

extern "C" int shim_eigenvalues(size_t ng, const size_t* n, double* const* a, double* const* w, int threads)
{
	return dmrgpp::group_eigenvalues(ng, n, a, w, g_red, threads) ? 0 : 1;
}

extern "C" void shim_vectors(size_t ng, const size_t* n, const size_t* k, const double* const* w, double* const* z,
                             int threads)
{
	dmrgpp::group_eigenvectors(ng, n, k, g_red.data(), w, z, threads);
	for (size_t g = 0; g < ng; ++g)
		if (n[g] >= 2 && k[g] > 0)
			dmrgpp::apply_q(int(n[g]), g_red[g].hv, g_red[g].beta, z[g], int(k[g]));
}
