// NVTX ranges around the library's entry points (NVTX v3, header-only).
// Without a profiler attached a range costs an indirect call; under one
// (Nsight Compute, Nsight Systems) each call shows as a named range on the
// host thread's timeline, and kernels can be filtered by it.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace dmrgpp {

class TraceRange {
public:
	explicit TraceRange(const char* name) { nvtxRangePushA(name); }
	~TraceRange() { nvtxRangePop(); }
	TraceRange(const TraceRange&)            = delete;
	TraceRange& operator=(const TraceRange&) = delete;
};

} // namespace dmrgpp

#define DMRGPP_TRACE_CAT2(a, b) a##b
#define DMRGPP_TRACE_CAT(a, b) DMRGPP_TRACE_CAT2(a, b)
// a range named `name` from here to the end of the enclosing scope
#define DMRGPP_TRACE(name) ::dmrgpp::TraceRange DMRGPP_TRACE_CAT(dmrgpp_trace_, __LINE__)(name)
