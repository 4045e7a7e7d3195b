// host_runtime_stub.cpp -- host-memory stand-ins for the four CUDA runtime
// calls the kites:: host graph classes make (cudaHostAlloc, cudaFreeHost,
// cudaMemcpy, cudaGetErrorString) and for the one C-ABI call of the error
// path, so that the host-side construction in include/kites/ can be built
// with g++ and checked on a machine without a GPU driver.  Page-locking does
// not matter to CPU reads and writes.  Test infrastructure only.
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

cudaError_t CUDARTAPI cudaMemcpy(void *dst, const void *src, size_t n, enum cudaMemcpyKind) {
  std::memcpy(dst, src, n);
  return cudaSuccess;
}

const char *CUDARTAPI cudaGetErrorString(cudaError_t) { return "host stand-in error"; }

const char *kites_last_error_string(void) { return ""; }

}  // extern "C"
