// cuda_error_check.cuh -- every failure becomes std::runtime_error, as in
// farkhor/KiTES kites/common/cuda_error_check.cuh:9-18; engine (C ABI)
// statuses go through the same path with the engine's message.
#ifndef KITES_B200_CUDA_ERROR_CHECK_CUH_
#define KITES_B200_CUDA_ERROR_CHECK_CUH_

#include <cuda_runtime.h>

#include <sstream>
#include <stdexcept>
#include <string>

#include "../../kites_b200.h"

#define CUDAErrorCheck(err) { ::kites::detail::cuda_assert((err), __FILE__, __LINE__); }
#define KITESErrorCheck(status) { ::kites::detail::kites_assert((status), __FILE__, __LINE__); }

namespace kites {
namespace detail {

inline void cuda_assert(cudaError_t err, const char *file, int line) {
  if (err != cudaSuccess) {
    std::ostringstream s;
    s << "CUDAAssert: " << cudaGetErrorString(err) << " " << file << " " << line << "\n";
    throw std::runtime_error(s.str());
  }
}

inline void kites_assert(int status, const char *file, int line) {
  if (status != KITES_OK) {
    std::ostringstream s;
    s << "kites engine error " << status << ": " << kites_last_error_string() << " "
      << file << " " << line << "\n";
    throw std::runtime_error(s.str());
  }
}

}  // namespace detail
}  // namespace kites

#endif
