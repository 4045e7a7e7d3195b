// host_runtime.cpp -- plain host-memory definitions of the four CUDA runtime
// calls that farkhor/KiTES's host buffers make on the CPU-only path
// (kites/memory/host_pinned_buffer.cuh:26-29,34-37,55-56 and
// kites/common/cuda_error_check.cuh:14).  Linking the reference's host code
// against these instead of libcudart lets its graph construction and its
// sanity_check loop run on a machine without a GPU driver; page-locking is
// irrelevant to CPU-side reads and writes, so the arithmetic is unchanged.
// TEST INFRASTRUCTURE ONLY (oracle/_ref).
#include <cuda_runtime_api.h>

#include <cstdlib>
#include <cstring>

extern "C" {

cudaError_t CUDARTAPI cudaHostAlloc(void **p, size_t size, unsigned int) {
  *p = std::aligned_alloc(64, (size + 63) / 64 * 64);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}

cudaError_t CUDARTAPI cudaFreeHost(void *p) {
  std::free(p);
  return cudaSuccess;
}

cudaError_t CUDARTAPI cudaMemcpy(void *dst, const void *src, size_t n,
                                 enum cudaMemcpyKind) {
  std::memcpy(dst, src, n);
  return cudaSuccess;
}

const char *CUDARTAPI cudaGetErrorString(cudaError_t) {
  return "host-memory runtime stand-in error";
}

}  // extern "C"
