// generic_kernels.cuh -- the pull iteration for user-supplied vertex
// programs (the four __host__ __device__ functions of README.md:14-24),
// instantiated in the caller's translation unit.  Same contract as the
// reference kernels (kites/device/kernels_single_device.cuh:18-426):
//   acc = initF(V[v]);  acc = redF(acc, nbrCompF(V[C[e]], &E[e])) over in-edges;
//   if updF(acc, V[v]) { V[v] = acc; set the flag; activate out-neighbours }.
// Built for sm_100a: one warp per 32 consecutive vertices (one frontier
// word), the warp's active in-edges merged into one range walked 32 at a
// time, owners found by a 5-step search over shared prefix sums, and a
// per-run reduction in shared memory; activation ORs whole words per run
// of equal target words.  Arbitrary redF means no atomics on V, so a hub
// row is walked by its one warp; the built-in operators of the C ABI use
// the edge-balanced kernels instead.
#ifndef KITES_B200_GENERIC_KERNELS_CUH_
#define KITES_B200_GENERIC_KERNELS_CUH_

#include <cuda_runtime.h>
#include <stdint.h>

namespace kites {
namespace generic {

constexpr int kWarps = 4;  // 128 threads per CTA

__device__ __forceinline__ uint32_t scan_incl(uint32_t x, uint32_t lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
    if (lane >= (uint32_t)d) x += y;
  }
  return x;
}

// Bounds of this lane's run of equal keys (keys non-decreasing per run).
__device__ __forceinline__ void run_bounds(uint32_t key, uint32_t lane, uint32_t *start,
                                           uint32_t *end, bool *head) {
  const uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, key, 1);
  *head = lane == 0 || prev != key;
  const uint32_t heads = __ballot_sync(0xFFFFFFFFu, *head);
  const uint32_t upto = 0xFFFFFFFFu >> (31u - lane);
  *start = 31u - __clz(heads & upto);
  const uint32_t later = heads & ~upto;
  *end = later ? (uint32_t)(__ffs(later) - 2) : 31u;
}

// The pull of one warp over its 32 consecutive vertices (this lane's vertex
// v, `active` its frontier test): every active vertex folds its in-edges
// with the user functions and stores the result when updF accepts it.
// Returns whether this lane's vertex was updated.  ex/beg/acc/part: the
// warp's 32-entry rows of shared scratch.
template <class vT, class eT, class OffT, class FInit, class FComp, class FRed, class FUpd>
__device__ __forceinline__ bool pull_warp(uint64_t v, bool active, uint32_t lane,
                                          const OffT *__restrict__ R,
                                          const uint32_t *__restrict__ C, vT *V, eT *E,
                                          uint32_t *ex, OffT *beg, vT *acc, vT *part,
                                          FInit &fInit, FComp &fComp, FRed &fRed, FUpd &fUpd) {
  uint32_t cnt = 0;
  vT old{};
  if (active) {
    const OffT b = R[v];
    cnt = (uint32_t)(R[v + 1] - b);
    beg[lane] = b;
    old = V[v];
    vT glob = old;
    fInit(acc[lane], glob);
  }
  const uint32_t incl = scan_incl(cnt, lane);
  const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
  ex[lane] = incl - cnt;
  __syncwarp();
  for (uint32_t base = 0; base < total; base += 32) {
    const uint32_t i = base + lane;
    uint32_t owner = 32u;
    if (i < total) {
      uint32_t j = 0;
#pragma unroll
      for (uint32_t step = 16; step; step >>= 1)
        if (ex[j + step] <= i) j += step;
      owner = j;
      const OffT e = beg[j] + (OffT)(i - ex[j]);
      fComp(part[lane], V[C[e]], E + e);
    }
    __syncwarp();
    uint32_t s, t;
    bool head;
    run_bounds(owner, lane, &s, &t, &head);
    if (head && owner < 32u)
      for (uint32_t k = s; k <= t; ++k) fRed(acc[owner], part[k]);
    __syncwarp();
  }
  bool upd = false;
  if (active) {
    upd = fUpd(acc[lane], old);
    if (upd) V[v] = acc[lane];
  }
  return upd;
}

template <class vT, class eT, class OffT, class FInit, class FComp, class FRed, class FUpd>
__global__ void __launch_bounds__(kWarps * 32)
    pull_iteration(uint64_t n, const OffT *__restrict__ R, const uint32_t *__restrict__ C,
                   vT *V, eT *E, uint32_t *flag, const uint32_t *__restrict__ rd, uint32_t *wr,
                   uint32_t shift, const OffT *__restrict__ actR,
                   const uint32_t *__restrict__ actC, FInit fInit, FComp fComp, FRed fRed,
                   FUpd fUpd) {
  __shared__ uint32_t ex_s[kWarps][32];
  __shared__ OffT beg_s[kWarps][32];
  __shared__ vT acc_s[kWarps][32];
  __shared__ vT part_s[kWarps][32];
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const uint64_t vb = ((uint64_t)blockIdx.x * kWarps + w) * 32;
  if (vb >= n) return;  // n is a multiple of 128: whole warps retire
  const uint64_t v = vb + lane;
  const uint32_t word = rd[(vb >> shift) >> 5];
  const bool active = (word >> ((v >> shift) & 31u)) & 1u;
  if (__ballot_sync(0xFFFFFFFFu, active) == 0) return;

  const bool upd = pull_warp<vT, eT, OffT>(v, active, lane, R, C, V, E, ex_s[w], beg_s[w],
                                           acc_s[w], part_s[w], fInit, fComp, fRed, fUpd);
  const uint32_t U = __ballot_sync(0xFFFFFFFFu, upd);
  if (U == 0) return;
  if (lane == 0) *flag = 1u;

  // Activation rows: the updated vertex (vpg == 1) or, for vpg > 1, the
  // first lane of each group with an updated vertex.
  const uint32_t vpg = 1u << shift;
  bool resp;
  uint64_t row;
  if (vpg == 1) {
    resp = upd;
    row = v;
  } else if (vpg < 32) {
    const uint32_t gmask = ((1u << vpg) - 1u) << (lane & ~(vpg - 1));
    resp = (lane & (vpg - 1)) == 0 && (U & gmask);
    row = v >> shift;
  } else {
    resp = lane == 0;
    row = vb >> shift;
  }
  uint32_t ocnt = 0;
  if (resp) {
    const OffT b = actR[row];
    ocnt = (uint32_t)(actR[row + 1] - b);
    beg_s[w][lane] = b;
  }
  const uint32_t oincl = scan_incl(ocnt, lane);
  const uint32_t ototal = __shfl_sync(0xFFFFFFFFu, oincl, 31);
  __syncwarp();
  ex_s[w][lane] = oincl - ocnt;
  __syncwarp();
  for (uint32_t base = 0; base < ototal; base += 32) {
    const uint32_t i = base + lane;
    uint32_t tw = 0xFFFFFFFFu, tb = 0;
    if (i < ototal) {
      uint32_t j = 0;
#pragma unroll
      for (uint32_t step = 16; step; step >>= 1)
        if (ex_s[w][j + step] <= i) j += step;
      const uint32_t tgt = actC[beg_s[w][j] + (OffT)(i - ex_s[w][j])];
      tw = tgt >> 5;
      tb = 1u << (tgt & 31u);
    }
    uint32_t s, t;
    bool head;
    run_bounds(tw, lane, &s, &t, &head);
    const uint32_t rm = (t == 31u ? 0xFFFFFFFFu : ((2u << t) - 1u)) & ~((1u << s) - 1u);
    const uint32_t bits = __reduce_or_sync(rm, tb);
    if (head && tw != 0xFFFFFFFFu) atomicOr(wr + tw, bits);
  }
}

// ---- mipmapped graphs: coarse activation ----------------------------------
// The frontier holds one bit per block of `cr` consecutive vertices.  Every
// vertex of an active block pulls; each block with an updated vertex gets
// its bit in `chg_blocks` (one atomicOr per distinct block per warp).
template <class vT, class eT, class FInit, class FComp, class FRed, class FUpd>
__global__ void __launch_bounds__(kWarps * 32)
    mip_pull_iteration(uint64_t n, const uint32_t *__restrict__ R,
                       const uint32_t *__restrict__ C, vT *V, eT *E, uint32_t *flag,
                       const uint32_t *__restrict__ rd, uint32_t cr, uint32_t *chg_blocks,
                       FInit fInit, FComp fComp, FRed fRed, FUpd fUpd) {
  __shared__ uint32_t ex_s[kWarps][32];
  __shared__ uint32_t beg_s[kWarps][32];
  __shared__ vT acc_s[kWarps][32];
  __shared__ vT part_s[kWarps][32];
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const uint64_t vb = ((uint64_t)blockIdx.x * kWarps + w) * 32;
  if (vb >= n) return;  // n is a multiple of 128: whole warps retire
  const uint64_t v = vb + lane;
  const uint32_t blk = (uint32_t)(v / cr);
  const bool active = (rd[blk >> 5] >> (blk & 31u)) & 1u;
  if (__ballot_sync(0xFFFFFFFFu, active) == 0) return;
  const bool upd = pull_warp<vT, eT, uint32_t>(v, active, lane, R, C, V, E, ex_s[w], beg_s[w],
                                               acc_s[w], part_s[w], fInit, fComp, fRed, fUpd);
  if (__ballot_sync(0xFFFFFFFFu, upd) == 0) return;
  if (lane == 0) *flag = 1u;
  const uint32_t peers = __match_any_sync(0xFFFFFFFFu, upd ? blk : 0xFFFFFFFFu);
  if (upd && (uint32_t)(__ffs(peers) - 1) == lane)
    atomicOr(chg_blocks + (blk >> 5), 1u << (blk & 31u));
}

constexpr uint32_t kMipRowsPerSlice = 256;  // block rows per grid row (multiple of 32)

// Next frontier: wr |= OR of the mipmap rows of the changed blocks.  The
// mipmap is row-major with `words` 32-bit words per row (mipmapDim / 32);
// a thread owns frontier word j over the kMipRowsPerSlice rows of its grid
// row, so its loads of row after row are coalesced across the warp.
__global__ void mip_expand(const uint32_t *__restrict__ mip, uint32_t words,
                           const uint32_t *__restrict__ chg_blocks, uint32_t *wr) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= words) return;
  const uint32_t b0 = blockIdx.y * kMipRowsPerSlice;
  const uint32_t b1 = min(b0 + kMipRowsPerSlice, words * 32u);
  uint32_t acc = 0;
  for (uint32_t b = b0; b < b1; b += 32) {
    uint32_t bits = chg_blocks[b >> 5];
    while (bits) {
      const uint32_t k = __ffs(bits) - 1;
      bits &= bits - 1;
      acc |= mip[(uint64_t)(b + k) * words + j];
    }
  }
  if (acc) atomicOr(wr + j, acc);
}

__global__ void clear_words(uint32_t *p, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = 0u;
}

}  // namespace generic
}  // namespace kites

#endif
