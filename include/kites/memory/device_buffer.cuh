// device_buffer.cuh -- device buffers of the kites:: API (farkhor/KiTES
// kites/memory/device_buffer.cuh:19-160).  A buffer either owns a
// cudaMalloc'd array, or is a non-owning view of an array the engine's pool
// owns (the arrays of a graph_csr_device).
#ifndef KITES_B200_DEVICE_BUFFER_CUH_
#define KITES_B200_DEVICE_BUFFER_CUH_

#include <cuda_runtime.h>

#include "../common/cuda_error_check.cuh"
#include "../device/stream.cuh"
#include "uva_buffer.cuh"

namespace kites {

template <typename T>
class device_buffer : public uva_buffer<T> {
  int residing_device_id = 0;
  bool owning = true;

  void construct(std::size_t n) {
    CUDAErrorCheck(cudaSetDevice(residing_device_id));
    CUDAErrorCheck(cudaMalloc((void **)&this->ptr, n * sizeof(T)));
    this->nElems = n;
  }

 public:
  device_buffer() = default;
  device_buffer(std::size_t n, int dev) : residing_device_id{dev} {
    if (n > 0) construct(n);
  }
  device_buffer(const uva_buffer<T> &src, int dev = 0) : device_buffer(src.size(), dev) {
    if (src.size())
      CUDAErrorCheck(cudaMemcpy(this->ptr, src.get_ptr(), src.sizeInBytes(), cudaMemcpyDefault));
  }
  // Non-owning view of engine memory.
  static device_buffer view(T *p, std::size_t n, int dev) {
    device_buffer b;
    b.ptr = p;
    b.nElems = n;
    b.residing_device_id = dev;
    b.owning = false;
    return b;
  }
  device_buffer(const device_buffer &) = delete;
  device_buffer &operator=(const device_buffer &) = delete;
  device_buffer(device_buffer &&o) noexcept
      : uva_buffer<T>{o.nElems, o.ptr}, residing_device_id{o.residing_device_id}, owning{o.owning} {
    o.nElems = 0;
    o.ptr = nullptr;
  }
  device_buffer &operator=(device_buffer &&o) noexcept {
    if (this != &o) {
      free();
      this->nElems = o.nElems;
      this->ptr = o.ptr;
      residing_device_id = o.residing_device_id;
      owning = o.owning;
      o.nElems = 0;
      o.ptr = nullptr;
    }
    return *this;
  }
  ~device_buffer() override { free(); }

  void free() override {
    if (this->nElems != 0 && owning) {
      cudaSetDevice(residing_device_id);
      cudaFree(this->ptr);
    }
    this->nElems = 0;
    this->ptr = nullptr;
  }
  virtual void alloc(std::size_t n, int dev = 0) {
    residing_device_id = dev;
    if (this->nElems == 0 && n > 0) construct(n);
  }
  int get_residing_device_id() const { return residing_device_id; }
  void reset() {
    CUDAErrorCheck(cudaSetDevice(residing_device_id));
    CUDAErrorCheck(cudaMemset((void *)this->ptr, 0, this->sizeInBytes()));
  }
  void reset(stream &ss) {
    CUDAErrorCheck(cudaSetDevice(residing_device_id));
    CUDAErrorCheck(cudaMemsetAsync((void *)this->ptr, 0, this->sizeInBytes(), ss.get()));
  }
};

class device_bitmap : public device_buffer<unsigned int> {
  std::size_t nBits = 0;

 public:
  device_bitmap() = default;
  device_bitmap(std::size_t n, int dev = 0)
      : device_buffer<unsigned int>((n + 31) / 32, dev), nBits{n} {}
  device_bitmap(device_buffer<unsigned int> &&b, std::size_t n)
      : device_buffer<unsigned int>(std::move(b)), nBits{n} {}
  void alloc(std::size_t n, int dev = 0) override {
    if (n > 0) nBits = n;
    device_buffer<unsigned int>::alloc((n + 31) / 32, dev);
  }
  std::size_t getnBits() const { return nBits; }
};

}  // namespace kites

#endif
