// trace_ranges.h -- NVTX ranges named after the reference's trace events.
//
// The reference logs the phases of a DSGD++ epoch as events "epoch",
// "subepoch", "computation", "communication", "barrier" and "loss"
// (mf/sgd/dsgdpp_impl.h:119,143,154,237,248,259; mf/sgd/sgd_impl.h:56-58,
// 101-108).  The library marks the same phases with NVTX ranges on the host
// thread that enqueues them, so a profiler's timeline shows them under those
// names.  NVTX 3 is header-only and costs a branch when no tool is attached.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace dsgdpp {

class TraceRange {
 public:
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

}  // namespace dsgdpp
