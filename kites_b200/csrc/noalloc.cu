// noalloc.cu -- single-source SSSP that allocates no device memory.
//
// Why it exists: some callers cannot allocate device memory at the moment
// they want a shortest-path answer -- for example code that reserves all of
// its memory at start-up and forbids allocation on its serving path, or a
// host whose device memory is owned by another runtime's allocator.  Such a
// caller hands over a graph and an output buffer it already owns; everything
// else this entry point needs (two frontier bitmaps and a 4-byte "something
// changed" flag) lives in the fixed array below, compiled into the library.
//
// The array is a file-scope __device__ variable: every GPU that loads the
// library holds kNoAllocScratchBytes (4 MiB + 256 B) of it until the process
// exits, whether or not this entry point is ever called.  In host code its
// name is only a stand-in, not a device address, so the address handed to
// the kernels comes from cudaGetSymbolAddress, looked up once per device
// (with that device current) by the first call on that device.  That first
// call should therefore come before any stream capture.
//
// Every call on a device shares the one array and it keeps the previous
// call's contents: each call clears the bitmaps and the flag before use, and
// calls that overlap on the GPU (different streams or host threads at once)
// race on it and must not be issued.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "kites_b200.h"

namespace kites_internal {
namespace {

// 256 B of flags, then two frontier bitmaps of up to 2^24 bits each.
constexpr uint64_t kNoAllocMaxVertices = 1ull << 24;
constexpr uint64_t kNoAllocHeader = 256;
constexpr uint64_t kNoAllocBitmapBytes = kNoAllocMaxVertices / 8;
constexpr uint64_t kNoAllocScratchBytes = kNoAllocHeader + 2 * kNoAllocBitmapBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNaWarps = 8;

// dist = INF, dist[source] = 0, both bitmaps and the flag cleared.
__global__ void k_na_init(uint32_t *dist, uint64_t n, uint32_t *bits, uint64_t words,
                          uint32_t *flag) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = tid; i < n; i += stride) dist[i] = kInf;
  for (uint64_t i = tid; i < 2 * words; i += stride) bits[i] = 0u;
  if (tid == 0) *flag = 0u;
}

// dist[source] = 0 and the frontier bit of every out-neighbour of source.
__global__ void k_na_seed(uint32_t *dist, uint32_t source, const uint32_t *__restrict__ outR,
                          const uint32_t *__restrict__ outC, uint32_t *frontier) {
  if (blockIdx.x == 0 && threadIdx.x == 0) dist[source] = 0u;
  for (uint32_t i = outR[source] + blockIdx.x * blockDim.x + threadIdx.x; i < outR[source + 1];
       i += gridDim.x * blockDim.x) {
    const uint32_t t = outC[i];
    atomicOr(frontier + (t >> 5), 1u << (t & 31u));
  }
}

// One pull iteration, one warp per frontier word: the active vertices'
// in-edges are merged into one range walked 32 at a time, each lane finds
// its row by a 5-step search over shared prefix sums, minima meet per row
// through __reduce_min_sync over runs of equal row, improved vertices are
// stored and their out-neighbours ORed into the next frontier.
__global__ void __launch_bounds__(kNaWarps * 32)
    k_na_pull(uint64_t n, const uint32_t *__restrict__ R, const uint32_t *__restrict__ C,
              const uint32_t *__restrict__ E, const uint32_t *__restrict__ outR,
              const uint32_t *__restrict__ outC, uint32_t *dist, const uint32_t *rd,
              uint32_t *wr, uint32_t *flag) {
  __shared__ uint32_t ex_s[kNaWarps][32];
  __shared__ uint32_t beg_s[kNaWarps][32];
  __shared__ uint32_t acc_s[kNaWarps][32];
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  const uint64_t words = (n + 31) / 32;
  for (uint64_t wi = (uint64_t)blockIdx.x * kNaWarps + w; wi < words;
       wi += (uint64_t)gridDim.x * kNaWarps) {
    const uint32_t word = rd[wi];
    if (word == 0) continue;
    const uint64_t v = wi * 32 + lane;
    const bool active = v < n && ((word >> lane) & 1u);
    uint32_t cnt = 0, old = kInf;
    if (active) {
      const uint32_t b = R[v];
      cnt = R[v + 1] - b;
      beg_s[w][lane] = b;
      old = dist[v];
    }
    acc_s[w][lane] = kInf;
    const uint32_t incl = warp_inclusive_scan(cnt);
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    ex_s[w][lane] = incl - cnt;
    __syncwarp();
    for (uint32_t base = 0; base < total; base += 32) {
      const uint32_t i = base + lane;
      uint32_t owner = 32u, p = kInf;
      if (i < total) {
        uint32_t j = 0;
#pragma unroll
        for (uint32_t step = 16; step; step >>= 1)
          if (ex_s[w][j + step] <= i) j += step;
        owner = j;
        const uint32_t e = beg_s[w][j] + (i - ex_s[w][j]);
        p = sat_add(dist[C[e]], E[e]);
      }
      bool head;
      const uint32_t rm = run_mask(owner, &head);
      const uint32_t q = __reduce_min_sync(rm, p);
      if (head && owner < 32u) acc_s[w][owner] = min(acc_s[w][owner], q);
      __syncwarp();
    }
    const bool upd = active && acc_s[w][lane] < old;
    if (upd) dist[v] = acc_s[w][lane];
    const uint32_t U = __ballot_sync(kFull, upd);
    if (U == 0) continue;
    if (lane == 0) *flag = 1u;
    // Activation: out-neighbours of the improved vertices.
    uint32_t ocnt = 0;
    __syncwarp();
    if (upd) {
      const uint32_t b = outR[v];
      ocnt = outR[v + 1] - b;
      beg_s[w][lane] = b;
    }
    const uint32_t oincl = warp_inclusive_scan(ocnt);
    const uint32_t ototal = __shfl_sync(kFull, oincl, 31);
    ex_s[w][lane] = oincl - ocnt;
    __syncwarp();
    for (uint32_t base = 0; base < ototal; base += 32) {
      const uint32_t i = base + lane;
      if (i < ototal) {
        uint32_t j = 0;
#pragma unroll
        for (uint32_t step = 16; step; step >>= 1)
          if (ex_s[w][j + step] <= i) j += step;
        const uint32_t t = outC[beg_s[w][j] + (i - ex_s[w][j])];
        atomicOr(wr + (t >> 5), 1u << (t & 31u));
      }
    }
    __syncwarp();
  }
}

// Caller graph check before any traversal: offsets start at 0, never
// decrease and end at the edge count; every id is below n.  Sets bits of
// *err instead of letting a bad index reach a gather or a bitmap write.
__global__ void k_na_validate(const uint32_t *__restrict__ R, const uint32_t *__restrict__ C,
                              uint64_t n, uint64_t m, uint32_t *err) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = tid; i < n; i += stride) {
    const uint32_t a = R[i], b = R[i + 1];
    if (a > b || (i == 0 && a != 0) || (i + 1 == n && (uint64_t)b != m)) atomicOr(err, 1u);
  }
  for (uint64_t i = tid; i < m; i += stride)
    if (C[i] >= n) atomicOr(err, 2u);
}

__global__ void k_na_clear(uint32_t *p, uint64_t words) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = 0u;
}

std::mutex g_na_mutex;
unsigned char *g_na_ptr[256];  // device address of g_noalloc_scratch, per device id

// Looks the array's device address up for the current device, once.
int noalloc_scratch(unsigned char **out) {
  int dev = -1;
  KITES_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) return fail(KITES_ERR_NO_DEVICE, "device id %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_ptr[dev]) {
    void *p = nullptr;
    KITES_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_na_ptr[dev] = (unsigned char *)p;
  }
  *out = g_na_ptr[dev];
  return KITES_OK;
}

}  // namespace
}  // namespace kites_internal

using namespace kites_internal;

extern "C" int kites_sssp_noalloc(const uint32_t *R, const uint32_t *C, const uint32_t *E,
                                  uint64_t n_edges, const uint32_t *out_R,
                                  const uint32_t *out_C, uint32_t n_vertices, uint32_t source,
                                  uint32_t *dist, void *stream, uint32_t *iterations) {
  clear_error();
  if (!R || !C || !E || !out_R || !out_C || !dist)
    return fail(KITES_ERR_INVALID, "null graph or output pointer");
  if (n_edges > 0xFFFFFFFFull) return fail(KITES_ERR_INVALID, "32-bit offsets: < 2^32 edges");
  if (n_vertices == 0 || (uint64_t)n_vertices > kNoAllocMaxVertices)
    return fail(KITES_ERR_INVALID,
                "kites_sssp_noalloc takes 1 .. %llu vertices (its fixed scratch holds two "
                "frontier bitmaps of that many bits); got %u",
                (unsigned long long)kNoAllocMaxVertices, n_vertices);
  if (source >= n_vertices) return fail(KITES_ERR_INVALID, "source %u out of range", source);
  unsigned char *scratch = nullptr;
  KITES_TRY(noalloc_scratch(&scratch));
  cudaStream_t s = (cudaStream_t)stream;
  const uint64_t n = n_vertices;
  const uint64_t words = (n + 31) / 32;
  uint32_t *flag = reinterpret_cast<uint32_t *>(scratch);
  uint32_t *err = flag + 1;
  uint32_t *bits = reinterpret_cast<uint32_t *>(scratch + kNoAllocHeader);
  uint32_t *frontier[2] = {bits, bits + words};
  KITES_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(uint32_t), s));
  k_na_validate<<<1184, 256, 0, s>>>(R, C, n, n_edges, err);
  k_na_validate<<<1184, 256, 0, s>>>(out_R, out_C, n, n_edges, err);
  uint32_t host_err = 0;
  KITES_CUDA_TRY(cudaMemcpyAsync(&host_err, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  KITES_CUDA_TRY(cudaStreamSynchronize(s));
  if (host_err & 1u)
    return fail(KITES_ERR_INVALID, "offsets are not 0 .. n_edges and non-decreasing");
  if (host_err & 2u) return fail(KITES_ERR_INVALID, "a vertex id is >= n_vertices");
  k_na_init<<<592, 256, 0, s>>>(dist, n, bits, words, flag);
  k_na_seed<<<32, 256, 0, s>>>(dist, source, out_R, out_C, frontier[0]);
  KITES_CUDA_TRY(cudaGetLastError());
  // Bellman-Ford-style pulls reach the fixed point within n + 1 rounds.
  const uint64_t cap = 2 * n + 16;
  uint64_t it = 0;
  uint32_t host_flag = 0;
  const unsigned grid = (unsigned)std::min<uint64_t>((words + kNaWarps - 1) / kNaWarps, 148 * 8);
  for (;;) {
    KITES_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(uint32_t), s));
    uint32_t *rd = frontier[it & 1], *wr = frontier[(it & 1) ^ 1];
    k_na_pull<<<grid, kNaWarps * 32, 0, s>>>(n, R, C, E, out_R, out_C, dist, rd, wr, flag);
    k_na_clear<<<(unsigned)std::min<uint64_t>((words + 255) / 256, 1184), 256, 0, s>>>(rd, words);
    KITES_CUDA_TRY(cudaGetLastError());
    KITES_CUDA_TRY(cudaMemcpyAsync(&host_flag, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    KITES_CUDA_TRY(cudaStreamSynchronize(s));
    ++it;
    if (host_flag == 0) break;
    if (it >= cap) {
      if (iterations) *iterations = (uint32_t)it;
      return fail(KITES_ERR_TIMEOUT, "no fixed point after %llu iterations",
                  (unsigned long long)it);
    }
  }
  if (iterations) *iterations = (uint32_t)it;
  return KITES_OK;
}
