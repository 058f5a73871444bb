// Every device allocation of the library goes through dev_alloc, so that a
// test can make one of them fail on the host (cupbr_debug_fail_allocation)
// and check that the call reports it and releases what it had allocated.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace cupbr_b200 {

// cudaMalloc, unless the injected failure is due: then nothing is
// allocated and cudaErrorMemoryAllocation is returned.
cudaError_t dev_alloc(void** p, size_t bytes);
template <typename T>
inline cudaError_t dev_alloc(T** p, size_t bytes) {
    return dev_alloc(reinterpret_cast<void**>(p), bytes);
}

// The n-th allocation from now (0: the next one) fails; n < 0: none does.
void dev_alloc_fail_after(int64_t n);

}  // namespace cupbr_b200
