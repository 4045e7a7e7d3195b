// nv_gpu.cuh -- one GPU of the kites:: API (farkhor/KiTES
// kites/device/nv_gpu.cuh:21-88), backed by an engine of the C ABI
// (kites_engine_create): the engine's stream is ssEven, on which every
// graph upload and every iteration runs.  The multi-GPU nv_gpus of the
// reference is not provided: this engine runs on one GPU.
#ifndef KITES_B200_NV_GPU_CUH_
#define KITES_B200_NV_GPU_CUH_

#include <cuda_runtime.h>

#include <utility>

#include "../../kites_b200.h"
#include "../common/cuda_error_check.cuh"
#include "stream.cuh"

namespace kites {

class nv_gpu {
  int devIdx;
  cudaDeviceProp devProp;
  kites_engine *eng = nullptr;
  kites::stream ssEven, ssOdd;

  static kites_engine *create(int idx) {
    kites_engine *e = nullptr;
    KITESErrorCheck(kites_engine_create(idx, &e));
    return e;
  }
  static cudaStream_t engine_stream(kites_engine *e) {
    void *s = nullptr;
    KITESErrorCheck(kites_engine_stream(e, &s));
    return (cudaStream_t)s;
  }

 public:
  explicit nv_gpu(int idx)
      : devIdx{idx}, eng{create(idx)}, ssEven{idx, engine_stream(eng)}, ssOdd{idx} {
    CUDAErrorCheck(cudaGetDeviceProperties(&devProp, idx));
    CUDAErrorCheck(cudaSetDevice(idx));
  }
  nv_gpu() : nv_gpu{0} {}
  nv_gpu(const nv_gpu &) = delete;
  nv_gpu &operator=(const nv_gpu &) = delete;
  nv_gpu &operator=(nv_gpu &&) = delete;
  nv_gpu(nv_gpu &&o) noexcept
      : devIdx{o.devIdx}, devProp(o.devProp), eng{o.eng}, ssEven{std::move(o.ssEven)},
        ssOdd{std::move(o.ssOdd)} {
    o.eng = nullptr;
  }
  ~nv_gpu() {
    if (eng) kites_engine_destroy(eng);
  }

  int getDevIdx() const { return devIdx; }
  cudaDeviceProp &getDevProp() { return devProp; }
  kites_engine *engine() const { return eng; }
  void setAsActive() const { CUDAErrorCheck(cudaSetDevice(devIdx)); }
  void sync() {
    setAsActive();
    CUDAErrorCheck(cudaDeviceSynchronize());
  }
  kites::stream &getSsEven() { return ssEven; }
  kites::stream &getSsOdd() { return ssOdd; }
  // (used MB, total MB) of device memory, as nv_gpu.cuh:78-86 reports it.
  std::pair<double, double> queryMemUsage() const {
    uint64_t used = 0, total = 0;
    KITESErrorCheck(kites_engine_mem_usage(eng, &used, &total, nullptr));
    return {used / 1000000.0, total / 1000000.0};
  }
};

// kites/device/compute.cuh:451-454
inline void sync_with(nv_gpu &d) { d.sync(); }

}  // namespace kites

#endif
