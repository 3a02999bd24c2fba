// fd3d_trace.h -- NVTX ranges around the C ABI's entry points, so that a timeline
// profiler shows which library call enqueued which kernels.  Header-only NVTX: without a
// profiler attached the calls return at once.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace fd3d {

struct TraceRange {
    explicit TraceRange(const char* name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};

}  // namespace fd3d
