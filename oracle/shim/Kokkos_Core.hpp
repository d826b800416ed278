// Host-only stand-in for the Kokkos names that the reference's CPU paths
// mention when compiled without Kokkos (the batched-GEMM path, PsimagLite's
// Lanczos solver, and PsimagLite's thread pool with one host execution
// space per thread).  Test infrastructure for the oracle build only.
#pragma once
#include <complex>
#include <vector>
namespace Kokkos {
struct DefaultExecutionSpace {};
template <class T> using complex = std::complex<T>;
inline void initialize(int&, char**) {}
inline void finalize() {}
struct ScopeGuard {
	ScopeGuard(int&, char**) {}
};
namespace Experimental {
template <class Space>
std::vector<Space> partition_space(const Space&, const std::vector<int>& weights)
{
	return std::vector<Space>(weights.size());
}
} // namespace Experimental
} // namespace Kokkos
