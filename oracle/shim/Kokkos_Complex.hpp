// Host-only stand-in for the three Kokkos names that the reference's CPU
// batched-GEMM path and PsimagLite's Lanczos solver mention when compiled
// without Kokkos.  Test infrastructure for the oracle build only.
#pragma once
#include <complex>
namespace Kokkos {
struct DefaultExecutionSpace {};
template <class T> using complex = std::complex<T>;
inline void initialize(int&, char**) {}
inline void finalize() {}
struct ScopeGuard {
	ScopeGuard(int&, char**) {}
};
} // namespace Kokkos
