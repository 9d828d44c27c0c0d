// Trace ranges around the C-ABI entry points: NVTX push/pop ranges named
// after the entry point, visible to Nsight Systems and to ncu's NVTX
// filters.  The NVTX v3 headers are header-only; without a tool attached a
// range costs a check of a null function pointer.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace go {

struct TraceRange {
    explicit TraceRange(const char* name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};

}  // namespace go

#define GO_TRACE(name) ::go::TraceRange go_trace_range_(name)
