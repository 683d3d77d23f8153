// sbx_trace.h — NVTX ranges around the host-side step sequence.
//
// NVTX v3 is header-only: with no tool attached every push/pop is a call that returns at
// once; a profiler that injects an NVTX tool (NVTX_INJECTION64_PATH) records the ranges.
// Names follow "sbx.<path>.<part>".
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace sbx {

struct TraceRange {
    explicit TraceRange(const char* name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};

// consecutive ranges in one scope: next() closes the open range and opens the next one
struct TracePhases {
    bool open = false;
    void next(const char* name) {
        if (open) nvtxRangePop();
        nvtxRangePushA(name);
        open = true;
    }
    TracePhases() = default;
    ~TracePhases() {
        if (open) nvtxRangePop();
    }
    TracePhases(const TracePhases&) = delete;
    TracePhases& operator=(const TracePhases&) = delete;
};

}  // namespace sbx

#define SBX_TRACE_CAT2(a, b) a##b
#define SBX_TRACE_CAT(a, b) SBX_TRACE_CAT2(a, b)
// a range from here to the end of the enclosing scope
#define SBX_TRACE(name) ::sbx::TraceRange SBX_TRACE_CAT(sbx_trace_, __LINE__)(name)
