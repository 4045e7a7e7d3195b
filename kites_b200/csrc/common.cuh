// common.cuh -- engine-internal types, error plumbing and warp primitives.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "kites_b200.h"
#include "status.h"

#define KITES_CUDA_TRY(call)                                                   \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess)                                                     \
      return kites_internal::fail(e_ == cudaErrorMemoryAllocation              \
                                      ? KITES_ERR_OOM                          \
                                      : KITES_ERR_CUDA,                        \
                                  "%s failed: %s (%s:%d)", #call,              \
                                  cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

#define KITES_TRY(expr)          \
  do {                           \
    int s_ = (expr);             \
    if (s_ != KITES_OK) return s_; \
  } while (0)

namespace kites_internal {

constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr uint32_t kInf = 0xFFFFFFFFu;
constexpr int kBlock = 256;          // threads per CTA of the traversal kernels
constexpr int kWarpsPerBlock = kBlock / 32;

// Built-in operators compiled into the library (kites_op).
enum : int { OP_SSSP = 0, OP_SSSP_WRAP = 1, OP_BFS = 2, OP_CC = 3, OP_PR = 4 };

// Device counters of one run: convergence state and per-iteration stats.
struct run_counters {
  uint32_t update_flag;     // set by any warp that updated a vertex
  uint32_t done;            // device loop: converged or out of iterations
  uint32_t timed_out;
  uint32_t pad0;
  unsigned long long iterations;
  unsigned long long max_iterations;
  unsigned long long active;          // active vertices, current iteration
  unsigned long long edges;           // in-edges of active vertices
  unsigned long long updated;         // vertices updated
  unsigned long long out_edges;       // activation edges visited
  unsigned long long total_active;
  unsigned long long total_edges;
  unsigned long long total_updated;
  unsigned long long total_out_edges;
  unsigned long long queue_len[2];    // compacted changed queue lengths
  unsigned long long last_active;     // active / edges of the previous iteration
  unsigned long long last_edges;
  unsigned long long last_out_edges;  // activation edges of the previous iteration
  unsigned long long changed;         // rows marked changed by the pull/push kernels
  unsigned long long last_changed;
  uint32_t sel;                       // strategy class picked for the next iteration
  uint32_t error;                     // kErr* bits: why a kernel stopped the run
};

// run_counters::error bits, set with atomicOr; any bit ends the loop.
constexpr uint32_t kErrIndex = 1u;    // an index read during the run was out of range
                                      // (the access was skipped)
constexpr uint32_t kErrWait = 2u;     // a bounded wait on a TMA copy gave up

__device__ __forceinline__ void raise_error(run_counters *c, uint32_t bit) {
  atomicOr(&c->error, bit);
}

// ---- warp primitives ---------------------------------------------------

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Inclusive warp scan of a 32-bit value with __shfl_up_sync.
__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t x) {
  const uint32_t lane = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(kFull, x, d);
    if (lane >= (uint32_t)d) x += y;
  }
  return x;
}

// Sum of a 64-bit value over the warp (every lane gets it).  Per-lane edge
// and degree counts can pass 2^32 on graphs with 64-bit offsets, so they
// are never narrowed before the reduction.
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
#pragma unroll
  for (int d = 16; d; d >>= 1) x += __shfl_xor_sync(kFull, x, d);
  return x;
}

// Mask of the lanes in the same run of equal `owner` values as this lane;
// owners are non-decreasing across the warp.
__device__ __forceinline__ uint32_t run_mask(uint32_t owner, bool *is_head) {
  const uint32_t lane = lane_id();
  uint32_t prev = __shfl_up_sync(kFull, owner, 1);
  bool head = (lane == 0) || (prev != owner);
  uint32_t heads = __ballot_sync(kFull, head);
  uint32_t upto = kFull >> (31u - lane);           // lanes 0..lane
  uint32_t start = 31u - __clz(heads & upto);
  uint32_t later = heads & ~upto;
  uint32_t end = later ? (uint32_t)(__ffs(later) - 2) : 31u;
  *is_head = head;
  uint32_t hi = (end == 31u) ? kFull : ((2u << end) - 1u);
  uint32_t lo = (1u << start) - 1u;
  return hi & ~lo;
}

__device__ __forceinline__ uint32_t sat_add(uint32_t a, uint32_t b) {
  uint32_t s = a + b;
  return s < a ? kInf : s;
}

template <int OP>
__device__ __forceinline__ uint32_t nbr_comp(uint32_t src, uint32_t w) {
  if (OP == OP_SSSP) return sat_add(src, w);
  if (OP == OP_SSSP_WRAP) return src + w;
  if (OP == OP_BFS) return src == kInf ? kInf : src + 1u;
  return src;  // OP_CC
}

template <int OP>
constexpr bool op_reads_weights() {
  return OP == OP_SSSP || OP == OP_SSSP_WRAP;
}

}  // namespace kites_internal
