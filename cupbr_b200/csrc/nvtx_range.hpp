// NVTX ranges around the library's host entry points and wavefront
// enqueues, so a timeline profiler shows which call issued which kernels.
// NVTX 3 is header only; without a profiler attached a range costs a
// branch on a null function pointer.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace cupbr_b200 {

struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace cupbr_b200
