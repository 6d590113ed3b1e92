// NVTX ranges around the entry points that enqueue GPU work (stepper launches, force
// evaluations, surrogate training and inference), named after the entry point, so that a
// timeline profiler shows the library's calls and ncu can select launches by range
// (--nvtx --nvtx-include).  NVTX v3 is header-only: with no tool attached a range costs a
// branch and nothing is recorded.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace bd {

class NvtxRange {
 public:
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace bd
