// generic_kernels.cuh -- the pull iteration for user-supplied vertex
// programs (the four __host__ __device__ functions of README.md:14-24),
// instantiated in the caller's translation unit.  Same contract as the
// reference kernels (kites/device/kernels_single_device.cuh:18-426):
//   acc = initF(V[v]);  acc = redF(acc, nbrCompF(V[C[e]], &E[e])) over in-edges;
//   if updF(acc, V[v]) { V[v] = acc; set the flag; activate out-neighbours }.
// redF is taken to be associative and commutative, as the reference's tree
// reduction over a warp's lanes already assumes; nothing else is assumed of
// it (no identity, no idempotence, no atomics on V).
//
// Layout, as the engine's built-in kernels: the CSC is cut into equal
// chunks of the item sequence "row v, then its in-edges" (the engine's
// chunk table), a warp owns a chunk at a time, so a hub row is spread over
// many warps instead of serialising one.  Inside a chunk the warp takes its
// rows 32 at a time, walks their in-edges 32 per step (owner of each edge by
// a 5-step search over shared prefix sums), and folds each step's values
// into their rows with a segmented warp-shuffle reduction using redF.  A
// row wholly inside the chunk is finished there; the parts of a row cut by
// chunk boundaries leave their folds in two per-chunk slots, and
// combine_split_rows joins them in chunk order, applies initF and updF, and
// stores the row.  Updated rows set their bit in the changed bitmap; the
// engine's activation (kites_graph_activate) turns it into the next
// frontier.
#ifndef KITES_B200_GENERIC_KERNELS_CUH_
#define KITES_B200_GENERIC_KERNELS_CUH_

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>

namespace kites {
namespace generic {

constexpr int kWarps = 4;  // 128 threads per CTA
constexpr uint32_t kFull = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t scan_incl(uint32_t x, uint32_t lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, x, d);
    if (lane >= (uint32_t)d) x += y;
  }
  return x;
}

// Bounds of this lane's run of equal keys (keys non-decreasing per run).
__device__ __forceinline__ void run_bounds(uint32_t key, uint32_t lane, uint32_t *start,
                                           uint32_t *end, bool *head) {
  const uint32_t prev = __shfl_up_sync(kFull, key, 1);
  *head = lane == 0 || prev != key;
  const uint32_t heads = __ballot_sync(kFull, *head);
  const uint32_t upto = kFull >> (31u - lane);
  *start = 31u - __clz(heads & upto);
  const uint32_t later = heads & ~upto;
  *end = later ? (uint32_t)(__ffs(later) - 2) : 31u;
}

// __shfl_down_sync of any trivially copyable value, 32 bits at a time.
template <class T>
__device__ __forceinline__ T shfl_down_any(const T &x, uint32_t d) {
  constexpr int W = (int)((sizeof(T) + 3) / 4);
  uint32_t w[W] = {};
  memcpy(w, &x, sizeof(T));
#pragma unroll
  for (int i = 0; i < W; ++i) w[i] = __shfl_down_sync(kFull, w[i], d);
  T y;
  memcpy(&y, w, sizeof(T));
  return y;
}

// Segmented warp reduction with the user's redF: lanes [start, end] form a
// run (equal owner); afterwards the run's first lane holds redF over the
// run's values.  Lane i ends holding the fold of [i, min(i + 31, end)].
template <class vT, class FRed>
__device__ __forceinline__ void fold_runs(vT &x, uint32_t lane, uint32_t end, FRed &fRed) {
#pragma unroll
  for (uint32_t d = 1; d < 32; d <<= 1) {
    vT y = shfl_down_any(x, d);
    if (lane + d <= end) fRed(x, y);
  }
}

// Folds nbrCompF over the in-edges of the warp's rows: lane j's row has
// cnt[j] edges starting at beg[j] (ex = exclusive prefix of the counts,
// total = their sum); the fold of row j lands in acc[j], has[j] says whether
// it holds any value (rows with no edges hold none).  kUnroll windows of 32
// edges have their values (the V[C[e]] gathers) in flight before any is
// reduced.
constexpr int kUnroll = 4;

template <class vT, class eT, class OffT, class FComp, class FRed>
__device__ __forceinline__ void fold_edges(uint32_t lane, uint32_t total, const uint32_t *ex,
                                           const OffT *beg, const uint32_t *__restrict__ C,
                                           const vT *V, eT *E, vT *acc, uint8_t *has,
                                           FComp &fComp, FRed &fRed) {
  for (uint32_t base = 0; base < total; base += 32 * kUnroll) {
    uint32_t owner[kUnroll];
    vT part[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const uint32_t i = base + u * 32 + lane;
      owner[u] = 32u;
      part[u] = vT{};
      if (i < total) {
        uint32_t j = 0;
#pragma unroll
        for (uint32_t step = 16; step; step >>= 1)
          if (ex[j + step] <= i) j += step;
        owner[u] = j;
        const OffT e = beg[j] + (OffT)(i - ex[j]);
        const vT src = V[C[e]];
        fComp(part[u], src, E + e);
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      uint32_t s, t;
      bool head;
      run_bounds(owner[u], lane, &s, &t, &head);
      fold_runs(part[u], lane, t, fRed);
      if (head && owner[u] < 32u) {
        if (has[owner[u]]) {
          fRed(acc[owner[u]], part[u]);
        } else {
          acc[owner[u]] = part[u];
          has[owner[u]] = 1;
        }
      }
      __syncwarp();
    }
  }
}

// ---- chunked pull -----------------------------------------------------------

// Device-side convergence state of one process() call.
struct loop_state {
  unsigned long long iterations, max_iterations;
  uint32_t done, timed_out;
};

template <class vT, class OffT>
struct chunk_args {
  const OffT *R;
  const uint32_t *C;
  const uint32_t *chunk_rows;   // row holding item k * chunk_items (n_chunks + 1 entries)
  uint64_t n_chunks, n_rows;
  uint32_t chunk_items;
  const uint32_t *rd;           // frontier (vertex or group bits)
  uint32_t *chg;                // changed rows (same bits)
  uint32_t shift;               // log2(vertex per group)
  uint32_t *flag;
  vT *part;                     // 2 slots per chunk: the first and the last row's fold
  uint8_t *part_has;
  const loop_state *ls;         // a finished loop skips the rest of its body
};

__device__ __forceinline__ bool bit_of(const uint32_t *bits, uint64_t v, uint32_t shift) {
  const uint64_t gi = v >> shift;
  return (bits[gi >> 5] >> (gi & 31u)) & 1u;
}

// Row v occupies items v + R[v] (the row) .. v + R[v + 1] (its last edge).
// In chunk ch it is whole when both ends lie there; a row cut by chunk
// boundaries leaves its part's fold in slot 2 ch when it is the chunk's
// first row, else (the chunk's last row) in slot 2 ch + 1.
template <class vT, class eT, class OffT, class FInit, class FComp, class FRed, class FUpd>
__global__ void __launch_bounds__(kWarps * 32)
    chunk_pull(chunk_args<vT, OffT> a, vT *V, eT *E, FInit fInit, FComp fComp, FRed fRed,
               FUpd fUpd) {
  if (a.ls->done) return;
  __shared__ uint32_t ex_s[kWarps][33];
  __shared__ OffT beg_s[kWarps][32];
  __shared__ vT acc_s[kWarps][32];
  __shared__ uint8_t has_s[kWarps][32];
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const uint64_t stride = (uint64_t)gridDim.x * kWarps;
  for (uint64_t ch = (uint64_t)blockIdx.x * kWarps + w; ch < a.n_chunks; ch += stride) {
    const uint64_t item_lo = ch * a.chunk_items, item_hi = item_lo + a.chunk_items;
    const uint64_t v_first = a.chunk_rows[ch];
    uint64_t v_last = a.chunk_rows[ch + 1];
    if (v_last >= a.n_rows) v_last = a.n_rows - 1;
    for (uint64_t vb = v_first & ~31ull; vb <= v_last; vb += 32) {
      const uint64_t v = vb + lane;
      bool active = v >= v_first && v <= v_last && bit_of(a.rd, v, a.shift);
      uint64_t r0 = 0, r1 = 0;
      if (active) {
        r0 = (uint64_t)a.R[v];
        r1 = (uint64_t)a.R[v + 1];
        active = v + r1 >= item_lo && v + r0 < item_hi;  // some item of v is here
      }
      if (__ballot_sync(kFull, active) == 0) continue;
      uint32_t cnt = 0;
      bool whole = false;
      if (active) {
        // Edge e of v is item v + 1 + e.
        const uint64_t lo = item_lo > v + 1 ? max(r0, item_lo - v - 1) : r0;
        const uint64_t hi = min(r1, item_hi - v - 1);
        cnt = hi > lo ? (uint32_t)(hi - lo) : 0u;
        beg_s[w][lane] = (OffT)lo;
        whole = v + r0 >= item_lo && v + r1 < item_hi;
      }
      has_s[w][lane] = 0;
      const uint32_t incl = scan_incl(cnt, lane);
      const uint32_t total = __shfl_sync(kFull, incl, 31);
      ex_s[w][lane] = incl - cnt;
      __syncwarp();
      fold_edges<vT, eT, OffT>(lane, total, ex_s[w], beg_s[w], a.C, V, E, acc_s[w], has_s[w],
                               fComp, fRed);
      bool upd = false;
      if (active && whole) {
        const vT old = V[v];
        vT glob = old, res;
        fInit(res, glob);
        if (has_s[w][lane]) fRed(res, acc_s[w][lane]);
        if (fUpd(res, old)) {
          V[v] = res;
          upd = true;
        }
      } else if (active) {
        const uint64_t slot = 2 * ch + (v == v_first ? 0u : 1u);
        a.part[slot] = acc_s[w][lane];
        a.part_has[slot] = has_s[w][lane];
      }
      __syncwarp();
      const uint32_t gbit = upd ? (1u << ((v >> a.shift) & 31u)) : 0u;
      const uint32_t bits = __reduce_or_sync(kFull, gbit);
      if (bits && lane == 0) {
        atomicOr(a.chg + ((vb >> a.shift) >> 5), bits);
        *a.flag = 1u;
      }
    }
  }
}

// One thread per chunk ch: the row r holding the first item past ch, if r
// starts in ch (so its later parts lie in the chunks after), is finished
// here: initF(V[r]) folded with its parts' slots in chunk order, then updF.
template <class vT, class eT, class OffT, class FInit, class FRed, class FUpd>
__global__ void combine_split_rows(chunk_args<vT, OffT> a, vT *V, FInit fInit, FRed fRed,
                                   FUpd fUpd) {
  if (a.ls->done) return;
  const uint64_t ch = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ch >= a.n_chunks) return;
  const uint64_t ci = a.chunk_items, item_lo = ch * ci, item_hi = item_lo + ci;
  const uint64_t r = a.chunk_rows[ch + 1];
  if (r >= a.n_rows) return;
  const uint64_t first = r + (uint64_t)a.R[r], last = r + (uint64_t)a.R[r + 1];
  if (first < item_lo || first >= item_hi || last < item_hi) return;  // not a row cut here
  if (!bit_of(a.rd, r, a.shift)) return;
  const vT old = V[r];
  vT glob = old, res;
  fInit(res, glob);
  uint64_t slot = 2 * ch + (a.chunk_rows[ch] == r ? 0u : 1u);
  for (uint64_t c = ch;;) {
    if (a.part_has[slot]) {
      vT p = a.part[slot];
      fRed(res, p);
    }
    ++c;
    if (c * ci > last) break;  // the row's last item lies in chunk c - 1
    slot = 2 * c;
  }
  if (fUpd(res, old)) {
    V[r] = res;
    const uint64_t gi = r >> a.shift;
    atomicOr(a.chg + (gi >> 5), 1u << (gi & 31u));
    *a.flag = 1u;
  }
}

// Ends the captured while loop when no row changed (the reference's host
// test of its flag, compute.cuh:122-128) or after max_iterations; counts
// iterations and clears the flag for the next one.  Once done, the rest of
// the loop body finds ls->done set and does nothing.
__global__ void loop_check(uint32_t *flag, loop_state *st, cudaGraphConditionalHandle h) {
  if (st->done) {
    cudaGraphSetConditional(h, 0);
    return;
  }
  const unsigned long long it = st->iterations + 1;
  st->iterations = it;
  bool stop = *flag == 0u;
  if (!stop && st->max_iterations && it >= st->max_iterations) {
    st->timed_out = 1u;
    stop = true;
  }
  *flag = 0u;
  if (stop) {
    st->done = 1u;
    cudaGraphSetConditional(h, 0);
  }
}

__global__ void clear_two(uint32_t *a, uint32_t *b, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    a[i] = 0u;
    b[i] = 0u;
  }
}

// ---- mipmapped graphs: coarse activation ----------------------------------
// The frontier holds one bit per block of `cr` consecutive vertices.  A warp
// takes 32 consecutive vertices; every vertex of an active block folds its
// in-edges (fold_edges) and each block with an updated vertex gets its bit
// in `chg_blocks` (one atomicOr per distinct block per warp).
template <class vT, class eT, class FInit, class FComp, class FRed, class FUpd>
__global__ void __launch_bounds__(kWarps * 32)
    mip_pull_iteration(uint64_t n, const uint32_t *__restrict__ R,
                       const uint32_t *__restrict__ C, vT *V, eT *E, uint32_t *flag,
                       const uint32_t *__restrict__ rd, uint32_t cr, uint32_t *chg_blocks,
                       FInit fInit, FComp fComp, FRed fRed, FUpd fUpd) {
  __shared__ uint32_t ex_s[kWarps][33];
  __shared__ uint32_t beg_s[kWarps][32];
  __shared__ vT acc_s[kWarps][32];
  __shared__ uint8_t has_s[kWarps][32];
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const uint64_t vb = ((uint64_t)blockIdx.x * kWarps + w) * 32;
  if (vb >= n) return;  // n is a multiple of 128: whole warps retire
  const uint64_t v = vb + lane;
  const uint32_t blk = (uint32_t)(v / cr);
  const bool active = (rd[blk >> 5] >> (blk & 31u)) & 1u;
  if (__ballot_sync(kFull, active) == 0) return;
  uint32_t cnt = 0;
  if (active) {
    beg_s[w][lane] = R[v];
    cnt = R[v + 1] - R[v];
  }
  has_s[w][lane] = 0;
  const uint32_t incl = scan_incl(cnt, lane);
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  ex_s[w][lane] = incl - cnt;
  __syncwarp();
  fold_edges<vT, eT, uint32_t>(lane, total, ex_s[w], beg_s[w], C, V, E, acc_s[w], has_s[w],
                               fComp, fRed);
  bool upd = false;
  if (active) {
    const vT old = V[v];
    vT glob = old, res;
    fInit(res, glob);
    if (has_s[w][lane]) fRed(res, acc_s[w][lane]);
    if (fUpd(res, old)) {
      V[v] = res;
      upd = true;
    }
  }
  if (__ballot_sync(kFull, upd) == 0) return;
  if (lane == 0) *flag = 1u;
  const uint32_t peers = __match_any_sync(kFull, upd ? blk : kFull);
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
