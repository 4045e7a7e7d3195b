// host_pinned_buffer.cuh -- page-locked host buffers and the host frontier
// bitmap of the kites:: API (farkhor/KiTES kites/memory/host_pinned_buffer.cuh:21-172):
// RAII, move-only, copy-constructible from any uva_buffer (device or host),
// bitmaps in 32-bit words with bit i of word w = element 32w + i.
#ifndef KITES_B200_HOST_PINNED_BUFFER_CUH_
#define KITES_B200_HOST_PINNED_BUFFER_CUH_

#include <cuda_runtime.h>

#include <cstring>
#include <ostream>
#include <stdexcept>

#include "../common/cuda_error_check.cuh"
#include "uva_buffer.cuh"

namespace kites {

template <typename T>
class host_pinned_buffer : public uva_buffer<T> {
  void construct(std::size_t n) {
    CUDAErrorCheck(cudaHostAlloc((void **)&this->ptr, n * sizeof(T), cudaHostAllocPortable));
    this->nElems = n;
  }

 public:
  host_pinned_buffer() = default;
  explicit host_pinned_buffer(std::size_t n) {
    if (n > 0) construct(n);
  }
  host_pinned_buffer(const uva_buffer<T> &src) : host_pinned_buffer(src.size()) {
    if (src.size())
      CUDAErrorCheck(cudaMemcpy(this->ptr, src.get_ptr(), src.sizeInBytes(), cudaMemcpyDefault));
  }
  host_pinned_buffer(const host_pinned_buffer &) = delete;
  host_pinned_buffer &operator=(const host_pinned_buffer &) = delete;
  host_pinned_buffer(host_pinned_buffer &&o) noexcept : uva_buffer<T>{o.nElems, o.ptr} {
    o.nElems = 0;
    o.ptr = nullptr;
  }
  host_pinned_buffer &operator=(host_pinned_buffer &&o) noexcept {
    if (this != &o) {
      free();
      this->nElems = o.nElems;
      this->ptr = o.ptr;
      o.nElems = 0;
      o.ptr = nullptr;
    }
    return *this;
  }
  ~host_pinned_buffer() override { free(); }

  void free() override {
    if (this->nElems != 0) {
      this->nElems = 0;
      cudaFreeHost(this->ptr);
      this->ptr = nullptr;
    }
  }
  virtual void alloc(std::size_t n) {
    if (this->nElems == 0 && n > 0) construct(n);
  }
  T &at(std::size_t i) {
    if (i >= this->nElems) throw std::runtime_error("The referred element does not exist in the buffer.");
    return this->ptr[i];
  }
  T &operator[](std::size_t i) { return this->ptr[i]; }
  const T &operator[](std::size_t i) const { return this->ptr[i]; }

  friend std::ostream &operator<<(std::ostream &os, host_pinned_buffer &b) {
    for (std::size_t i = 0; i < b.size(); ++i) os << b.at(i) << "\n";
    return os;
  }
};

class host_bitmap : public host_pinned_buffer<unsigned int> {
  std::size_t nBits = 0;

 public:
  host_bitmap() = default;
  explicit host_bitmap(std::size_t n) : host_pinned_buffer<unsigned int>((n + 31) / 32), nBits{n} {}
  void alloc(std::size_t n) override {
    if (n > 0) nBits = n;
    host_pinned_buffer<unsigned int>::alloc((n + 31) / 32);
  }
  void setAt(std::size_t pos) { this->ptr[pos >> 5] |= (1u << (pos & 31)); }
  bool getAt(std::size_t pos) const { return (this->ptr[pos >> 5] >> (pos & 31)) & 1u; }
  void reset() {
    if (this->nElems) std::memset(this->ptr, 0, this->sizeInBytes());
  }
  std::size_t getnBits() const { return nBits; }
  unsigned int count() const {
    unsigned int c = 0;
    for (std::size_t i = 0; i < this->size(); ++i) c += __builtin_popcount(this->ptr[i]);
    return c;
  }
};

}  // namespace kites

#endif
