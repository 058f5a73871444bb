// Host stand-ins for the three CUDA runtime calls that the reference's
// object-BVH constructor and Memory helpers make (lib/src/Core/MemoryDetail.h:
// cudaMalloc/cudaFree/cudaMemcpy).  Linked ONLY into oracle/_ref/libref_host.so,
// where the reference's __host__ __device__ code is compiled with g++ so that
// its own BVH build (BoundingVolumeHierarchy.cpp:46-136) produces a tree of
// host pointers that its own traversal can walk on the CPU.  Test
// infrastructure; never part of the product.
#include <cuda_runtime_api.h>
#include <cstdlib>
#include <cstring>

extern "C" {

cudaError_t cudaMalloc(void** ptr, size_t size) {
    *ptr = std::malloc(size ? size : 1);
    return *ptr ? cudaSuccess : cudaErrorMemoryAllocation;
}

cudaError_t cudaFree(void* ptr) {
    std::free(ptr);
    return cudaSuccess;
}

cudaError_t cudaMemcpy(void* dst, const void* src, size_t count, enum cudaMemcpyKind) {
    std::memcpy(dst, src, count);
    return cudaSuccess;
}

}  // extern "C"
