// Host-only stand-in for Kokkos profiling regions (oracle build only).
#pragma once
#include <string>
namespace Kokkos {
namespace Profiling {
struct ScopedRegion {
	explicit ScopedRegion(const std::string&) {}
};
inline void pushRegion(const std::string&) {}
inline void popRegion() {}
} // namespace Profiling
} // namespace Kokkos
