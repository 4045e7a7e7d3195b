// uva_buffer.cuh -- the abstract buffer interface of the kites:: API
// (farkhor/KiTES kites/memory/uva_buffer.cuh:14-52): element count, a
// pointer valid under unified virtual addressing, and free().
#ifndef KITES_B200_UVA_BUFFER_CUH_
#define KITES_B200_UVA_BUFFER_CUH_

#include <cstddef>

namespace kites {

template <typename T>
class uva_buffer {
 protected:
  std::size_t nElems = 0;
  T *ptr = nullptr;

 public:
  uva_buffer() = default;
  uva_buffer(std::size_t n, T *p) : nElems{n}, ptr{p} {}
  T *get_ptr() const { return ptr; }
  std::size_t size() const { return nElems; }
  std::size_t sizeInBytes() const { return nElems * sizeof(T); }
  virtual void free() = 0;
  virtual ~uva_buffer() {}
};

}  // namespace kites

#endif
