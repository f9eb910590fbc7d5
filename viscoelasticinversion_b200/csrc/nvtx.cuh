// nvtx.cuh — NVTX ranges around the host-side phases (a time step call, the
// gradient's forward sweep / recompute / adjoint sweep, a batch run, a
// served slice), so a timeline profiler shows where a run spends its time.
// NVTX v3 is header-only: with no profiler attached a range costs a branch.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace vb {

struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

}  // namespace vb
