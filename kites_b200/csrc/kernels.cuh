// kernels.cuh -- sm_100a kernels of the built-in vertex programs.
//
// Layout.  The CSC (rows = destinations, kites/graph/graph_csr.h:28-39) is
// split once, at upload, into equal chunks of the merged sequence
// "vertex v, then its in-edges" (item position of v is v + R[v], of edge e
// of v is v + 1 + e).  A warp owns one chunk at a time, so every warp does
// the same number of items whatever the degree skew; a hub's row simply
// spans several chunks and its partial minima meet through atomicMin.
//
// Iteration (the reference's pull kernel, kernels_single_device.cuh:18-426,
// re-designed):
//   k_pull_chunked    active vertices (bit of the read frontier) reduce
//                     nbrComp(V[C[e]], E[e]) over their in-edges with a
//                     warp-segmented min (__reduce_min_sync over runs of
//                     equal owner), update V in place and mark the
//                     vertex/group in the `changed` bitmap;
//   k_expand_chunked  for each changed row of the activation adjacency
//                     (dir_R/dir_C, or C for undirected graphs) set the
//                     out-neighbour bits of the write frontier;
//   memset            clears the read frontier and the changed bitmap
//                     (compute.cuh:121);
//   k_loop_check      counts the iteration and ends the loop when no vertex
//                     changed (compute.cuh:122-128), on the device.
#pragma once
#include "common.cuh"

namespace kites_internal {

// ---- chunk table ------------------------------------------------------------

// chunk_v0[k] = largest row r with r + R[r] <= k * chunk_items (k <= nchunks).
template <typename OffT>
__global__ void k_chunk_table(const OffT *__restrict__ R, uint64_t n_rows,
                              uint64_t nchunks, uint32_t chunk_items,
                              uint32_t *__restrict__ chunk_v0) {
  uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k > nchunks) return;
  const uint64_t target = k * chunk_items;
  uint64_t lo = 0, hi = n_rows;  // answer in [0, n_rows)
  while (hi - lo > 1) {
    uint64_t mid = (lo + hi) >> 1;
    if (mid + (uint64_t)R[mid] <= target) lo = mid; else hi = mid;
  }
  chunk_v0[k] = (uint32_t)lo;
}

template <typename OffT>
struct chunk_geom {
  const OffT *R;
  const uint32_t *C;
  const uint32_t *chunk_v0;
  uint64_t nchunks;
  uint64_t n_rows;
  uint64_t n_items;
  uint32_t chunk_items;
};

// ---- pull -------------------------------------------------------------------

constexpr int kUnroll = 4;  // 32-edge windows in flight per warp

// Per-warp row slice of one chunk: lanes hold (count, first edge) of their
// row's edges inside the chunk; ex = exclusive prefix of the counts.
template <typename OffT>
struct row_slice {
  uint32_t *ex;
  OffT *lo;
};

// Owner lane of virtual edge i (largest j with ex[j] <= i; a lane with no
// edges shares its ex with the next lane, so the search lands on a lane
// that owns edges).
__device__ __forceinline__ uint32_t owner_of(const uint32_t *ex, uint32_t i) {
  uint32_t j = 0;
#pragma unroll
  for (uint32_t step = 16; step; step >>= 1)
    if (ex[j + step] <= i) j += step;
  return j;
}

// Folds p(e) over the slice's `total` virtual edges into acc[owner] with a
// warp-segmented min.  The policy splits each edge into a streaming load
// (C, and E when needed) and a dependent value (the V gather), so kUnroll
// windows of both are in flight before any reduction.
template <typename OffT, class Policy>
__device__ __forceinline__ void fold_min(const row_slice<OffT> &rs, uint32_t total,
                                         uint32_t *acc, const Policy &pol) {
  const uint32_t lane = lane_id();
  for (uint32_t base = 0; base < total; base += 32 * kUnroll) {
    uint32_t own[kUnroll], c[kUnroll], w[kUnroll], p[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const uint32_t i = base + u * 32 + lane;
      own[u] = 32u;
      c[u] = 0u;
      w[u] = 0u;
      if (i < total) {
        const uint32_t j = owner_of(rs.ex, i);
        own[u] = j;
        pol.load(rs.lo[j] + (OffT)(i - rs.ex[j]), &c[u], &w[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) p[u] = own[u] < 32u ? pol.value(c[u], w[u]) : kInf;
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      bool head;
      const uint32_t rm = run_mask(own[u], &head);
      const uint32_t q = __reduce_min_sync(rm, p[u]);
      if (head && own[u] < 32u) acc[own[u]] = min(acc[own[u]], q);
      __syncwarp();
    }
  }
}

// Edge policies.  PullEdges: every in-edge of an active row.
template <int OP>
struct pull_edges {
  const uint32_t *C, *E, *V;
  __device__ __forceinline__ void load(uint64_t e, uint32_t *c, uint32_t *w) const {
    *c = __ldcs(C + e);
    if (op_reads_weights<OP>()) *w = __ldcs(E + e);
  }
  __device__ __forceinline__ uint32_t value(uint32_t c, uint32_t w) const {
    return nbr_comp<OP>(V[c], w);
  }
};

// FilteredEdges: only in-edges whose source changed last iteration (bit in U).
template <int OP>
struct filtered_edges {
  const uint32_t *C, *E, *V, *U;
  __device__ __forceinline__ void load(uint64_t e, uint32_t *c, uint32_t *w) const {
    const uint32_t src = __ldcs(C + e);
    const bool on = (U[src >> 5] >> (src & 31u)) & 1u;
    *c = on ? src : kInf;
    if (op_reads_weights<OP>() && on) *w = E[e];
  }
  __device__ __forceinline__ uint32_t value(uint32_t c, uint32_t w) const {
    return c == kInf ? kInf : nbr_comp<OP>(V[c], w);
  }
};

template <typename OffT>
struct pull_args {
  chunk_geom<OffT> g;
  const uint32_t *E;
  uint32_t *V;
  const uint32_t *rd;      // read frontier (bit per vertex or per group); null = all rows
  uint32_t *chg;           // changed rows of the activation adjacency
  uint32_t shift;          // log2(vertex_per_group)
  run_counters *ctr;
  const uint32_t *U;       // filtered pull: changed set of the previous iteration
  // Density gate: 0 always run; 1 run only while the frontier is sparse (the
  // staged sweep takes dense frontiers).  Dense = activation edges (this
  // iteration's when gate_cur, else the previous one's) above dense_edges.
  uint32_t gate, gate_cur;
  unsigned long long dense_edges;
  // PLAIN with the fused dense step: when the previous iteration's changed
  // rows exceed fused_rows (0 = off), k_sweep_changed pulls from them and
  // this kernel has nothing to do.
  unsigned long long fused_rows;
};

__device__ __forceinline__ bool frontier_dense(const run_counters *c, uint32_t cur,
                                               unsigned long long dense_edges) {
  return (cur ? c->out_edges : c->last_out_edges) > dense_edges;
}

// The pull iteration over the edge-balanced chunks.  Rows whose frontier
// bit is set (every row when rd is null) fold their in-edges with the edge
// policy; a row entirely inside the chunk stores its new value, a row split
// over chunks merges through atomicMin; updated rows set their bit (vertex
// or group) in chg.
// Whether any bitmap word in [w0, w1] is non-zero: four independent loads
// per round trip (a loop that stops at the first live word would wait for
// each load before issuing the next).
__device__ __forceinline__ bool any_word(const uint32_t *bits, uint64_t w0, uint64_t w1) {
  for (uint64_t w = w0; w <= w1; w += 4) {
    uint32_t x = bits[w];
    if (w + 1 <= w1) x |= bits[w + 1];
    if (w + 2 <= w1) x |= bits[w + 2];
    if (w + 3 <= w1) x |= bits[w + 3];
    if (x) return true;
  }
  return false;
}

template <int OP, typename OffT, bool kFiltered>
__device__ __forceinline__ void pull_chunks(const pull_args<OffT> &a) {
  __shared__ uint32_t s_ex[kWarpsPerBlock][32];
  __shared__ OffT s_lo[kWarpsPerBlock][32];
  __shared__ uint32_t s_acc[kWarpsPerBlock][32];
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  const row_slice<OffT> rs{s_ex[wib], s_lo[wib]};
  uint32_t *acc_s = s_acc[wib];
  uint32_t n_act = 0, n_edges = 0, n_chg = 0;
  const uint64_t stride = (uint64_t)gridDim.x * kWarpsPerBlock;
  // Warp gw owns chunks gw, gw + W, gw + 2W, ... (W warps in the grid), 32
  // of them per round: lane l tests whether the round's l-th chunk has any
  // frontier bit (a short run of words), and only those chunks are walked --
  // a sparse frontier costs one round trip per 32 chunks instead of a walk
  // of every chunk.
  const uint64_t gw = (uint64_t)blockIdx.x * kWarpsPerBlock + wib;
  for (uint64_t cbase = gw; cbase < a.g.nchunks; cbase += stride * 32) {
    bool live_chunk = false;
    {
      const uint64_t c = cbase + (uint64_t)lane * stride;
      if (c < a.g.nchunks) {
        if (!a.rd) {
          live_chunk = true;
        } else {
          const uint64_t v0 = a.g.chunk_v0[c];
          uint64_t v1 = a.g.chunk_v0[c + 1];
          if (v1 >= a.g.n_rows) v1 = a.g.n_rows - 1;
          live_chunk = any_word(a.rd, (v0 >> a.shift) >> 5, (v1 >> a.shift) >> 5);
        }
      }
    }
    uint32_t live_mask = __ballot_sync(kFull, live_chunk);
    while (live_mask) {
      const uint64_t ch = cbase + (uint64_t)(__ffs(live_mask) - 1) * stride;
      live_mask &= live_mask - 1;
      const int64_t item_lo = (int64_t)(ch * a.g.chunk_items);
      const int64_t item_hi =
          min(item_lo + (int64_t)a.g.chunk_items, (int64_t)a.g.n_items);
      const uint64_t v_first = a.g.chunk_v0[ch];
      uint64_t v_last = a.g.chunk_v0[ch + 1];
      if (v_last >= a.g.n_rows) v_last = a.g.n_rows - 1;
      for (uint64_t vb = v_first & ~31ull; vb <= v_last; vb += 32) {
        const uint64_t v = vb + lane;
        const bool in_range = v >= v_first && v <= v_last;
        bool active = in_range;
        if (a.rd) {
          const uint32_t word = a.rd[(vb >> a.shift) >> 5];
          active = in_range && ((word >> ((v >> a.shift) & 31u)) & 1u);
        }
        if (__ballot_sync(kFull, active) == 0) continue;
        uint32_t cnt = 0, old = 0;
        OffT elo = 0;
        bool whole = false;
        if (active) {
          const int64_t r0 = (int64_t)a.g.R[v], r1 = (int64_t)a.g.R[v + 1];
          const int64_t lo = max(r0, item_lo - (int64_t)v - 1);
          const int64_t hi = min(r1, item_hi - (int64_t)v - 1);
          cnt = hi > lo ? (uint32_t)(hi - lo) : 0u;
          elo = (OffT)lo;
          whole = (lo == r0) && (hi == r1);
          const int64_t vpos = (int64_t)v + r0;
          n_act += (vpos >= item_lo && vpos < item_hi) ? 1u : 0u;
          n_edges += cnt;
          if (cnt) old = a.V[v];
        }
        const uint32_t incl = warp_inclusive_scan(cnt);
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        if (total == 0) continue;
        rs.ex[lane] = incl - cnt;
        rs.lo[lane] = elo;
        acc_s[lane] = kInf;
        __syncwarp();
        if (kFiltered)
          fold_min(rs, total, acc_s, filtered_edges<OP>{a.g.C, a.E, a.V, a.U});
        else
          fold_min(rs, total, acc_s, pull_edges<OP>{a.g.C, a.E, a.V});
        bool upd = false;
        if (cnt) {
          const uint32_t acc = acc_s[lane];
          if (acc < old) {
            if (whole) {
              a.V[v] = acc;
              upd = true;
            } else {
              upd = acc < atomicMin(a.V + v, acc);
            }
          }
        }
        __syncwarp();
        const uint32_t gbit = upd ? (1u << ((v >> a.shift) & 31u)) : 0u;
        const uint32_t bits = __reduce_or_sync(kFull, gbit);
        if (bits && lane == 0) {
          const uint32_t old = atomicOr(a.chg + ((vb >> a.shift) >> 5), bits);
          n_chg += __popc(bits & ~old);
          a.ctr->update_flag = 1u;
        }
      }
    }
  }
  n_act = __reduce_add_sync(kFull, n_act);
  n_edges = __reduce_add_sync(kFull, n_edges);
  if (lane == 0) {
    if (n_act) atomicAdd(&a.ctr->active, (unsigned long long)n_act);
    if (n_edges) atomicAdd(&a.ctr->edges, (unsigned long long)n_edges);
    if (n_chg) atomicAdd(&a.ctr->changed, (unsigned long long)n_chg);
  }
}

template <int OP, typename OffT>
__global__ void __launch_bounds__(kBlock) k_pull_chunked(pull_args<OffT> a) {
  if (a.ctr->done) return;
  if (a.gate == 1 && frontier_dense(a.ctr, a.gate_cur, a.dense_edges)) return;
  if (a.fused_rows && a.ctr->last_changed > a.fused_rows) return;
  pull_chunks<OP, OffT, false>(a);
}

// ---- activation -------------------------------------------------------------

template <typename OffT>
struct expand_args {
  chunk_geom<OffT> g;      // rows of the activation adjacency
  const uint32_t *chg;     // changed rows
  uint32_t *wr;            // write frontier
  run_counters *ctr;
  // Gate: 0 always run; 1 only while the changed set is sparse (the pull
  // activation k_activate_sweep takes dense ones).  Dense = changed rows (this
  // iteration's when gate_cur, else the previous one's) above dense_rows.
  uint32_t gate, gate_cur;
  unsigned long long dense_rows;
};

__device__ __forceinline__ bool changed_dense(const run_counters *c, uint32_t cur,
                                              unsigned long long dense_rows) {
  return (cur ? c->changed : c->last_changed) > dense_rows;
}

// For each changed row, OR the bit of every target into the write frontier;
// lanes hitting the same target word in a window combine their bits first.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_expand_chunked(expand_args<OffT> a) {
  if (a.ctr->done) return;
  if (a.gate == 1 && changed_dense(a.ctr, a.gate_cur, a.dense_rows)) return;
  __shared__ uint32_t s_ex[kWarpsPerBlock][32];
  __shared__ OffT s_lo[kWarpsPerBlock][32];
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  uint32_t *ex = s_ex[wib];
  OffT *lo_s = s_lo[wib];
  uint32_t n_rows = 0, n_edges = 0;
  const uint64_t stride = (uint64_t)gridDim.x * kWarpsPerBlock;
  // Warp gw owns chunks gw, gw + W, gw + 2W, ...; per round each lane tests
  // one of the next 32 for a changed row and only those chunks are walked
  // (a sparse changed set costs one round trip per 32 chunks, not one per
  // bitmap word of every chunk).
  const uint64_t gw = (uint64_t)blockIdx.x * kWarpsPerBlock + wib;
  for (uint64_t cbase = gw; cbase < a.g.nchunks; cbase += stride * 32) {
    bool live_chunk = false;
    {
      const uint64_t c = cbase + (uint64_t)lane * stride;
      if (c < a.g.nchunks) {
        const uint64_t v0 = a.g.chunk_v0[c];
        uint64_t v1 = a.g.chunk_v0[c + 1];
        if (v1 >= a.g.n_rows) v1 = a.g.n_rows - 1;
        live_chunk = any_word(a.chg, v0 >> 5, v1 >> 5);
      }
    }
    uint32_t live_mask = __ballot_sync(kFull, live_chunk);
    while (live_mask) {
      const uint64_t ch = cbase + (uint64_t)(__ffs(live_mask) - 1) * stride;
      live_mask &= live_mask - 1;
      const int64_t item_lo = (int64_t)(ch * a.g.chunk_items);
      const int64_t item_hi =
          min(item_lo + (int64_t)a.g.chunk_items, (int64_t)a.g.n_items);
      const uint64_t r_first = a.g.chunk_v0[ch];
      uint64_t r_last = a.g.chunk_v0[ch + 1];
      if (r_last >= a.g.n_rows) r_last = a.g.n_rows - 1;
      for (uint64_t rb = r_first & ~31ull; rb <= r_last; rb += 32) {
        const uint32_t word = a.chg[rb >> 5];
        if (word == 0) continue;
        const uint64_t r = rb + lane;
        const bool active =
            r >= r_first && r <= r_last && ((word >> lane) & 1u);
        uint32_t cnt = 0;
        OffT elo = 0;
        if (active) {
          const int64_t r0 = (int64_t)a.g.R[r], r1 = (int64_t)a.g.R[r + 1];
          const int64_t lo = max(r0, item_lo - (int64_t)r - 1);
          const int64_t hi = min(r1, item_hi - (int64_t)r - 1);
          cnt = hi > lo ? (uint32_t)(hi - lo) : 0u;
          elo = (OffT)lo;
          const int64_t rpos = (int64_t)r + r0;
          n_rows += (rpos >= item_lo && rpos < item_hi) ? 1u : 0u;
          n_edges += cnt;
        }
        const uint32_t incl = warp_inclusive_scan(cnt);
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        if (total == 0) continue;
        ex[lane] = incl - cnt;
        lo_s[lane] = elo;
        __syncwarp();
        for (uint32_t base = 0; base < total; base += 32 * kUnroll) {
          uint32_t t[kUnroll];
#pragma unroll
          for (int u = 0; u < kUnroll; ++u) {
            const uint32_t i = base + u * 32 + lane;
            t[u] = kFull;
            if (i < total) {
              const uint32_t j = owner_of(ex, i);
              t[u] = __ldcs(a.g.C + lo_s[j] + (OffT)(i - ex[j]));
            }
          }
#pragma unroll
          for (int u = 0; u < kUnroll; ++u) {
            const uint32_t tword = t[u] == kFull ? kFull : (t[u] >> 5);
            const uint32_t tbit = t[u] == kFull ? 0u : (1u << (t[u] & 31u));
            bool head;
            const uint32_t rm = run_mask(tword, &head);
            const uint32_t bits = __reduce_or_sync(rm, tbit);
            if (head && tword != kFull) atomicOr(a.wr + tword, bits);
          }
        }
        __syncwarp();
      }
    }
  }
  n_rows = __reduce_add_sync(kFull, n_rows);
  n_edges = __reduce_add_sync(kFull, n_edges);
  if (lane == 0) {
    if (n_rows) atomicAdd(&a.ctr->updated, (unsigned long long)n_rows);
    if (n_edges) atomicAdd(&a.ctr->out_edges, (unsigned long long)n_edges);
  }
}

// ---- loop control -----------------------------------------------------------

// Per-iteration bookkeeping, one thread.  With a conditional-node handle it
// also ends the captured while loop (device-side convergence).
struct iter_record {
  unsigned long long *active;
  unsigned long long *edges;
  uint32_t capacity;
};

__global__ void k_loop_check(run_counters *c, iter_record rec,
                             cudaGraphConditionalHandle handle, int has_handle) {
  if (c->done) {
    if (has_handle) cudaGraphSetConditional(handle, 0);
    return;
  }
  const unsigned long long it = c->iterations;
  if (it < rec.capacity) {
    if (rec.active) rec.active[it] = c->active;
    if (rec.edges) rec.edges[it] = c->edges;
  }
  c->iterations = it + 1;
  c->last_active = c->active;
  c->last_edges = c->edges;
  c->last_out_edges = c->out_edges;
  c->last_changed = c->changed;
  c->changed = 0;
  c->queue_len[0] = 0;
  c->total_active += c->active;
  c->total_edges += c->edges;
  c->total_updated += c->updated;
  c->total_out_edges += c->out_edges;
  c->active = c->edges = c->updated = c->out_edges = 0;
  bool stop = false;
  if (c->update_flag == 0 || c->error) {
    stop = true;
  } else {
    c->update_flag = 0;
    if (c->max_iterations && c->iterations >= c->max_iterations) {
      c->timed_out = 1;
      stop = true;
    }
  }
  if (stop) {
    c->done = 1;
    if (has_handle) cudaGraphSetConditional(handle, 0);
  }
}

// ---- initialisation ---------------------------------------------------------

__global__ void k_fill_u32(uint32_t *p, uint64_t n, uint32_t value) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = value;
}

__global__ void k_iota_u32(uint32_t *p, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = (uint32_t)i;
}

// Sets V[source] = 0 and the frontier bit of every out-neighbour group of
// `source` (the example's pre-processing: bit d/vpg for each edge source->d).
template <typename OffT>
__global__ void k_seed_source(uint32_t *V, const OffT *__restrict__ outR,
                              const uint32_t *__restrict__ outC, uint32_t source,
                              uint32_t shift, uint32_t *frontier) {
  if (blockIdx.x == 0 && threadIdx.x == 0) V[source] = 0u;
  const OffT b = outR[source], e = outR[source + 1];
  for (OffT i = b + (OffT)(blockIdx.x * blockDim.x + threadIdx.x); i < e;
       i += (OffT)(gridDim.x * blockDim.x)) {
    const uint32_t g = outC[i] >> shift;
    atomicOr(frontier + (g >> 5), 1u << (g & 31u));
  }
}

// Every bit in [0, nbits) set, the rest of the words 0.
__global__ void k_all_active(uint32_t *bits, uint64_t nbits, uint64_t nwords) {
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nwords;
       w += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = w * 32;
    uint32_t m = 0;
    if (lo + 32 <= nbits) m = kFull;
    else if (lo < nbits) m = (1u << (uint32_t)(nbits - lo)) - 1u;
    bits[w] = m;
  }
}

// Upload validation: R[0] == 0, R non-decreasing, R[n_rows] == n_edges, and
// every id of `ids` below `limit`.  Any violation sets *bad; nothing is
// traversed before these pass, so a malformed graph is an error status,
// never an out-of-range access.
template <typename OffT>
__global__ void k_validate_rows(const OffT *__restrict__ R, uint64_t n_rows,
                                uint64_t n_edges, uint32_t *bad) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_rows;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const OffT a = R[i], b = R[i + 1];
    if (a > b || (i == 0 && a != 0) || (i + 1 == n_rows && (uint64_t)b != n_edges))
      atomicOr(bad, 1u);
  }
}

__global__ void k_validate_ids(const uint32_t *__restrict__ ids, uint64_t n,
                               uint64_t limit, uint32_t *bad) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    if (ids[i] >= limit) atomicOr(bad, 2u);
}

// Zeroes `words` words (read frontier + changed bitmap of one parity).
__global__ void k_clear_words(uint32_t *p, uint64_t words) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = 0u;
}

// R[n_src+1 .. n_rows] = R[n_src]: empty rows for the 128-padding vertices.
template <typename OffT>
__global__ void pad_offsets(OffT *R, uint64_t n_src, uint64_t n_rows) {
  const OffT last = R[n_src];
  for (uint64_t i = n_src + 1 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
       i <= n_rows; i += (uint64_t)gridDim.x * blockDim.x)
    R[i] = last;
}

// ---- out-CSR transposition helpers -------------------------------------------

template <typename OffT>
__global__ void k_row_of_edge(const OffT *__restrict__ R, uint64_t n_rows,
                              uint64_t n_edges, uint32_t *__restrict__ row) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n_edges;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = 0, hi = n_rows;  // largest r with R[r] <= e
    while (hi - lo > 1) {
      uint64_t mid = (lo + hi) >> 1;
      if ((uint64_t)R[mid] <= e) lo = mid; else hi = mid;
    }
    row[e] = (uint32_t)lo;
  }
}

__global__ void k_count_u32(const uint32_t *__restrict__ keys, uint64_t n,
                            uint32_t *__restrict__ counts) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(counts + keys[i], 1u);
}

template <typename OffT>
__global__ void k_gather_out(const uint32_t *__restrict__ order,
                             const uint32_t *__restrict__ row_of_edge,
                             const uint32_t *__restrict__ E, uint64_t n,
                             uint32_t *__restrict__ outC, uint32_t *__restrict__ outE) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t e = order[i];
    outC[i] = row_of_edge[e];
    if (outE) outE[i] = E ? E[e] : 1u;
  }
}

template <typename OffT>
__global__ void k_widen_offsets(const uint32_t *__restrict__ in, uint64_t n,
                                OffT *__restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (OffT)in[i];
}

template <typename OffT>
__global__ void k_narrow_offsets(const uint64_t *__restrict__ in, uint64_t n,
                                 OffT *__restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (OffT)in[i];
}

}  // namespace kites_internal
