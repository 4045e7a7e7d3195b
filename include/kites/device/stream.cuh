// stream.cuh -- CUDA stream wrapper of the kites:: API (farkhor/KiTES
// kites/device/stream.cuh:12-61); may also wrap, without owning, the
// stream of the engine.
#ifndef KITES_B200_STREAM_CUH_
#define KITES_B200_STREAM_CUH_

#include <cuda_runtime.h>

#include "../common/cuda_error_check.cuh"

namespace kites {

class stream {
  int residing_device_id = 0;
  cudaStream_t strm = nullptr;
  bool owning = true;

 public:
  stream() = delete;
  explicit stream(int dev) : residing_device_id{dev} {
    CUDAErrorCheck(cudaSetDevice(dev));
    CUDAErrorCheck(cudaStreamCreate(&strm));
  }
  stream(int dev, cudaStream_t borrowed) : residing_device_id{dev}, strm{borrowed}, owning{false} {}
  stream(const stream &) = delete;
  stream &operator=(const stream &) = delete;
  stream &operator=(stream &&) = delete;
  stream(stream &&o) noexcept
      : residing_device_id{o.residing_device_id}, strm{o.strm}, owning{o.owning} {
    o.strm = nullptr;
  }
  ~stream() {
    if (strm != nullptr && owning) {
      cudaSetDevice(residing_device_id);
      cudaStreamDestroy(strm);
    }
  }
  void sync() {
    CUDAErrorCheck(cudaSetDevice(residing_device_id));
    CUDAErrorCheck(cudaStreamSynchronize(strm));
  }
  cudaStream_t &get() { return strm; }
  cudaStream_t *get_ptr() { return &strm; }
  int getResidingDeviceId() const { return residing_device_id; }
};

}  // namespace kites

#endif
