// NVTX ranges around the host steps of the verify path (admission, packing,
// launches, copies back, RLC rounds), so that a timeline tool shows where a
// call spends its time next to its kernels.  The NVTX v3 headers are
// header-only and call nothing until a tool attaches itself, so the ranges
// cost a branch when no tool runs.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace uf {

struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace uf
