// mem_ops.cuh -- copyMem / copyMemOnStream of the kites:: API (farkhor/KiTES
// kites/memory/mem_ops.cuh:16-88): copies between any two uva_buffers;
// the synchronous form returns its wall time in milliseconds.
#ifndef KITES_B200_MEM_OPS_CUH_
#define KITES_B200_MEM_OPS_CUH_

#include <algorithm>
#include <chrono>

#include "../common/globals.cuh"
#include "../device/stream.cuh"
#include "device_buffer.cuh"
#include "host_pinned_buffer.cuh"

namespace kites {

// launch::sync blocks and returns the copy's wall time in ms; launch::async
// enqueues the copy on the default stream and returns 0 at once (the caller
// synchronises), as the reference's overload does.
template <class T, launch lMode = launch::sync>
double copyMem(uva_buffer<T> &dst, uva_buffer<T> &src, std::size_t length,
               std::size_t dstOffst = 0, std::size_t srcOffst = 0) {
  if (lMode == launch::async) {
    CUDAErrorCheck(cudaMemcpyAsync(dst.get_ptr() + dstOffst, src.get_ptr() + srcOffst,
                                   length * sizeof(T), cudaMemcpyDefault));
    return 0;
  }
  auto t0 = std::chrono::steady_clock::now();
  CUDAErrorCheck(cudaMemcpy(dst.get_ptr() + dstOffst, src.get_ptr() + srcOffst,
                            length * sizeof(T), cudaMemcpyDefault));
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

template <class T, launch lMode = launch::sync>
double copyMem(uva_buffer<T> &dst, uva_buffer<T> &src, std::size_t dstOffst = 0,
               std::size_t srcOffst = 0) {
  return copyMem<T, lMode>(dst, src, std::min(src.size(), dst.size()), dstOffst, srcOffst);
}

template <class T>
void copyMemOnStream(uva_buffer<T> &dst, uva_buffer<T> &src, std::size_t length, stream &s,
                     std::size_t dstOffst = 0, std::size_t srcOffst = 0) {
  CUDAErrorCheck(cudaMemcpyAsync(dst.get_ptr() + dstOffst, src.get_ptr() + srcOffst,
                                 length * sizeof(T), cudaMemcpyDefault, s.get()));
}

template <class T>
void copyMemOnStream(uva_buffer<T> &dst, uva_buffer<T> &src, stream &s,
                     std::size_t dstOffst = 0, std::size_t srcOffst = 0) {
  copyMemOnStream(dst, src, std::min(src.size(), dst.size()), s, dstOffst, srcOffst);
}

}  // namespace kites

#endif
