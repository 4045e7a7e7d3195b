// kites.cuh -- umbrella header of the kites:: API (farkhor/KiTES
// kites/kites.cuh:4-14): #include "kites/kites.cuh" and link
// libkites_b200.so.  Single-GPU only: the multi-device graph classes of
// the reference are not provided.
#ifndef KITES_B200_KITES_CUH_
#define KITES_B200_KITES_CUH_

#include "common/globals.cuh"
#include "common/cuda_error_check.cuh"
#include "memory/host_pinned_buffer.cuh"
#include "memory/device_buffer.cuh"
#include "memory/mem_ops.cuh"
#include "device/stream.cuh"
#include "device/nv_gpu.cuh"
#include "graph/graph_csr.h"
#include "graph/graph_csr_device.cuh"
#include "graph/graph_csr_mipmapped.hpp"
#include "graph/graph_csr_mipmapped_device.cuh"
#include "device/compute.cuh"
#include "io/graph_output.cuh"
#include "graph/sanity_check.cuh"

#endif
