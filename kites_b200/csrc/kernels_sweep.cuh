// kernels_sweep.cuh -- the tiled dense sweep over the CSC.
//
// For iterations where most rows (or most sources) are live, walking the
// CSC tile by tile beats per-row discovery.  A tile is kTileItems
// consecutive items of the merged "row, then its in-edges" sequence (row v
// at item v + R[v], its edge e at v + 1 + e).  A CTA first marks the tile's
// vertex items in a shared bitmap (one bit per item) and records each row's
// local position; then every warp walks 8 windows of 32 consecutive items,
// one item per lane.  A lane's row is the number of vertex items up to it
// (prefix popcounts of the bitmap), its edge index follows from the row, so
// the loads of C and E are coalesced and every lane has all of its gathers
// in flight together.  Row minima meet in a shared accumulator through the
// warp-segmented min (runs of equal row) and shared atomicMin; rows that
// lie wholly in the tile store their value, rows split across tiles merge
// into V with global atomicMin.
//
// Modes: kRowFilter -- rows whose frontier bit is set (PLAIN on a dense
// frontier); kEdgeFilter -- every row, only in-edges whose source changed
// last iteration (PULL_ALL).  k_expand_sweep is the same walk over the
// activation adjacency.
#pragma once
#include "kernels.cuh"

namespace kites_internal {

constexpr int kSweepThreads = 256;
constexpr int kSweepWarps = kSweepThreads / 32;
constexpr int kWindows = 8;                                   // windows of 32 items per warp
constexpr int kTileItems = kSweepWarps * kWindows * 32;       // 2048
constexpr int kTileWords = kTileItems / 32;                   // vertex-item bitmap words
constexpr int kRowSlots = kTileItems + 4;                     // rows + 1 <= 2050
constexpr int kFrontierWords = 72;                            // bitmap words of <= 2049 rows

enum { kRowFilter = 0, kEdgeFilter = 1 };

template <typename OffT>
struct sweep_args {
  const OffT *R;
  const uint32_t *C;
  const uint32_t *E;
  uint32_t *V;
  const uint32_t *tile_v0;   // chunk table with kTileItems items per chunk
  uint64_t ntiles, n_rows, n_items;
  const uint32_t *rd;        // kRowFilter: frontier bits (expand: the changed rows)
  const uint32_t *U;         // kEdgeFilter: changed bits of the previous iteration
  uint32_t *chg;             // next changed bits (expand: the frontier written)
  run_counters *ctr;
  uint64_t m;                // edges
  // Density gate (see pull_args / expand_args): 2 = run only when dense.
  uint32_t gate, gate_cur;
  unsigned long long dense_edges;
};

// Shared memory of a sweep CTA (static, < 17 KB).
struct sweep_smem {
  int32_t pos[kRowSlots];       // local position of row j's vertex item
  uint32_t acc[kRowSlots];      // row minima
  uint32_t isv[kTileWords];     // bit i: item i is a vertex item
  uint32_t fw[kFrontierWords];  // frontier / changed words of the rows
};

struct tile_geom {
  uint64_t item_lo, v0;
  uint32_t rows, nloc;          // rows v0 .. v0 + rows - 1; items [item_lo, item_lo + nloc)
};

template <typename OffT>
__device__ __forceinline__ tile_geom tile_of(const sweep_args<OffT> &a, uint64_t t) {
  tile_geom g;
  g.item_lo = t * (uint64_t)kTileItems;
  g.nloc = (uint32_t)(min(g.item_lo + (uint64_t)kTileItems, a.n_items) - g.item_lo);
  g.v0 = a.tile_v0[t];
  uint64_t v1 = a.tile_v0[t + 1];
  if (v1 >= a.n_rows) v1 = a.n_rows - 1;
  g.rows = (uint32_t)(v1 - g.v0 + 1);
  return g;
}

// Phase A: pos[j] = v0 + j + R[v0 + j] - item_lo for j in [0, rows], clamped
// to [-1, kTileItems + 1] (outside the tile only "before" and "after"
// matter: only row 0 starts before it, only row `rows` after it); the
// bitmap bit of every vertex item inside the tile; acc = INF; the rows'
// bitmap words from `bits` (when given).  isv must be zero on entry.
template <typename OffT>
__device__ __forceinline__ void tile_setup(const sweep_args<OffT> &a, const tile_geom &g,
                                           const uint32_t *bits, sweep_smem &sm) {
  for (uint32_t j = threadIdx.x; j <= g.rows; j += kSweepThreads) {
    const int64_t p = (int64_t)(g.v0 + j) + (int64_t)a.R[g.v0 + j] - (int64_t)g.item_lo;
    sm.pos[j] = (int32_t)max((int64_t)-1, min(p, (int64_t)kTileItems + 1));
    if (p >= 0 && p < (int64_t)g.nloc) atomicOr(&sm.isv[p >> 5], 1u << (p & 31));
    if (j < g.rows) sm.acc[j] = kInf;
  }
  if (bits) {
    const uint32_t nw = ((uint32_t)(g.v0 & 31u) + g.rows + 31u) >> 5;  // <= 66
    for (uint32_t i = threadIdx.x; i < nw; i += kSweepThreads) sm.fw[i] = bits[(g.v0 >> 5) + i];
  }
}

// Per-warp view of the tile: window k of warp w covers items
// (w * kWindows + k) * 32 + lane.  row(item) = vertex items up to and
// including it, minus 1 when the tile starts with row v0's vertex item.
struct window_rows {
  uint32_t pfx[kWindows];  // vertex items before each window
  uint32_t adj;
  __device__ __forceinline__ window_rows(const sweep_smem &sm) {
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    const uint32_t c0 = __popc(sm.isv[lane]), c1 = __popc(sm.isv[lane + 32]);
    const uint32_t s0 = warp_inclusive_scan(c0), s1 = warp_inclusive_scan(c1);
    const uint32_t t0 = __shfl_sync(kFull, s0, 31);
    const uint32_t ex0 = s0 - c0, ex1 = t0 + s1 - c1;
#pragma unroll
    for (int k = 0; k < kWindows; ++k) {
      const uint32_t wi = w * kWindows + k;  // warp-uniform
      pfx[k] = __shfl_sync(kFull, wi < 32 ? ex0 : ex1, wi & 31u);
    }
    adj = sm.pos[0] == 0 ? 1u : 0u;
  }
};

template <int OP, typename OffT, int MODE>
__global__ void __launch_bounds__(kSweepThreads, 4) k_sweep(sweep_args<OffT> a) {
  if (a.ctr->done) return;
  if (a.gate == 2 && !frontier_dense(a.ctr, a.gate_cur, a.dense_edges)) return;
  constexpr bool kW = op_reads_weights<OP>();
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  __shared__ sweep_smem sm;
  const uint32_t tid = threadIdx.x, lane = lane_id(), w = tid >> 5;
  const uint32_t le_mask = kFull >> (31u - lane);  // lanes 0 .. lane
  uint32_t n_act = 0, n_edges = 0, n_chg = 0;
  if (tid < kTileWords) sm.isv[tid] = 0u;
  __syncthreads();
  for (uint64_t t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const tile_geom g = tile_of(a, t);
    tile_setup(a, g, MODE == kRowFilter ? a.rd : nullptr, sm);
    __syncthreads();
    const window_rows wr(sm);
    const uint32_t vb = (uint32_t)(g.v0 & 31u);
    const int64_t ebase = (int64_t)g.item_lo - (int64_t)g.v0 - 1;  // e = ebase + xi - row
    // Rows and edge indices of the warp's 8 windows, then every load of the
    // windows before any use: C and E, the changed-source words, V.
    uint32_t row[kWindows], src[kWindows], wt[kWindows];
    uint64_t e[kWindows];
    bool live[kWindows];
#pragma unroll
    for (int k = 0; k < kWindows; ++k) {
      const uint32_t wi = w * kWindows + k;
      const uint32_t xi = wi * 32 + lane;
      const uint32_t word = sm.isv[wi];
      row[k] = kNone;
      live[k] = false;
      e[k] = 0;
      if (xi < g.nloc) {
        row[k] = wr.pfx[k] + __popc(word & le_mask) - wr.adj;
        const bool vertex = (word >> lane) & 1u;
        bool on = true;
        if (MODE == kRowFilter) {
          const uint32_t b = vb + row[k];
          on = (sm.fw[b >> 5] >> (b & 31u)) & 1u;
        }
        if (!vertex && on) {
          const int64_t ei = ebase + (int64_t)xi - (int64_t)row[k];
          if (ei < 0 || ei >= (int64_t)a.m || row[k] >= g.rows) {
            a.ctr->error = 1u;  // geometry out of step: never index with it
          } else {
            e[k] = (uint64_t)ei;
            live[k] = true;
          }
        }
      }
    }
    // PULL_ALL reads E only for edges from a changed source.
    constexpr bool kEarlyE = kW && MODE == kRowFilter;
#pragma unroll
    for (int k = 0; k < kWindows; ++k) {
      src[k] = live[k] ? __ldcs(a.C + e[k]) : 0u;
      wt[k] = (kEarlyE && live[k]) ? __ldcs(a.E + e[k]) : 0u;
    }
#pragma unroll
    for (int k = 0; k < kWindows; ++k)
      if (live[k] && src[k] >= a.n_rows) {
        a.ctr->error = 1u;
        live[k] = false;
      }
    if (MODE == kEdgeFilter) {
      uint32_t uw[kWindows];
#pragma unroll
      for (int k = 0; k < kWindows; ++k) uw[k] = live[k] ? a.U[src[k] >> 5] : 0u;
#pragma unroll
      for (int k = 0; k < kWindows; ++k)
        live[k] = live[k] && ((uw[k] >> (src[k] & 31u)) & 1u);
    }
    uint32_t val[kWindows];
#pragma unroll
    for (int k = 0; k < kWindows; ++k) {
      if (kW && !kEarlyE) wt[k] = live[k] ? __ldcs(a.E + e[k]) : 0u;
      val[k] = live[k] ? a.V[src[k]] : kInf;
    }
#pragma unroll
    for (int k = 0; k < kWindows; ++k) {
      const uint32_t cand = live[k] ? nbr_comp<OP>(val[k], wt[k]) : kInf;
      n_edges += live[k] ? 1u : 0u;
      bool head;
      const uint32_t rm = run_mask(row[k], &head);
      const uint32_t q = __reduce_min_sync(rm, cand);
      if (head && q != kInf) atomicMin(&sm.acc[row[k]], q);
    }
    __syncthreads();
    // Finalise the tile's rows.  A row whose items all lie in the tile has
    // this CTA as its only writer; a split row merges with atomicMin.
    if (tid < kTileWords) sm.isv[tid] = 0u;  // ready for the next tile
    for (uint32_t jb = 0; jb < g.rows; jb += kSweepThreads) {
      const uint32_t j = jb + tid;
      bool upd = false;
      if (j < g.rows) {
        const uint32_t acc = sm.acc[j];
        const int32_t p0 = sm.pos[j];
        if (acc != kInf) {
          const uint64_t v = g.v0 + j;
          const bool whole = p0 >= 0 && sm.pos[j + 1] <= (int32_t)g.nloc;
          const uint32_t old = a.V[v];
          if (acc < old) upd = whole ? (a.V[v] = acc, true) : (acc < atomicMin(a.V + v, acc));
        }
        if (MODE == kRowFilter) {
          const uint32_t b = vb + j;
          if ((sm.fw[b >> 5] >> (b & 31u)) & 1u)
            n_act += (p0 >= 0 && p0 < (int32_t)g.nloc) ? 1u : 0u;
        }
      }
      // Vertices of 32 consecutive rows share at most two words; the second
      // word is touched only when it receives bits (of vertices < n).
      const uint64_t wv = g.v0 + jb + (tid & ~31u);
      const uint32_t off = (uint32_t)(wv & 31u);
      const uint32_t bal = __ballot_sync(kFull, upd);
      if (bal && lane == 0) {
        const uint32_t lo = bal << off, hi = off ? (bal >> (32u - off)) : 0u;
        if (lo) n_chg += __popc(lo & ~atomicOr(a.chg + (wv >> 5), lo));
        if (hi) n_chg += __popc(hi & ~atomicOr(a.chg + (wv >> 5) + 1, hi));
        a.ctr->update_flag = 1u;
      }
    }
    __syncthreads();
  }
  n_act = __reduce_add_sync(kFull, n_act);
  n_edges = __reduce_add_sync(kFull, n_edges);
  n_chg = __reduce_add_sync(kFull, n_chg);
  if (lane == 0) {
    if (n_act) atomicAdd(&a.ctr->active, (unsigned long long)n_act);
    if (n_edges) atomicAdd(&a.ctr->edges, (unsigned long long)n_edges);
    if (n_chg) atomicAdd(&a.ctr->changed, (unsigned long long)n_chg);
  }
}

// Dense activation: the same walk over the activation adjacency (rows =
// changed candidates, C = targets); every edge of a row whose bit is set in
// rd (the changed rows) ORs its target's bit into chg (the frontier being
// written), lanes hitting one word in a window combining their bits first.
// gate: 2 = run only when the changed set is dense (see expand_args).
template <typename OffT>
__global__ void __launch_bounds__(kSweepThreads) k_expand_sweep(sweep_args<OffT> a) {
  if (a.ctr->done) return;
  if (a.gate == 2 && !changed_dense(a.ctr, a.gate_cur, a.dense_edges)) return;
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  __shared__ sweep_smem sm;
  const uint32_t tid = threadIdx.x, lane = lane_id(), w = tid >> 5;
  const uint32_t le_mask = kFull >> (31u - lane);
  uint32_t n_rows = 0, n_edges = 0;
  if (tid < kTileWords) sm.isv[tid] = 0u;
  __syncthreads();
  for (uint64_t t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const tile_geom g = tile_of(a, t);
    tile_setup(a, g, a.rd, sm);
    __syncthreads();
    const window_rows wr(sm);
    const uint32_t vb = (uint32_t)(g.v0 & 31u);
    const int64_t ebase = (int64_t)g.item_lo - (int64_t)g.v0 - 1;
    uint32_t tgt[kWindows];
#pragma unroll
    for (int k = 0; k < kWindows; ++k) {
      const uint32_t wi = w * kWindows + k;
      const uint32_t xi = wi * 32 + lane;
      const uint32_t word = sm.isv[wi];
      tgt[k] = kNone;
      if (xi >= g.nloc) continue;
      const uint32_t r = wr.pfx[k] + __popc(word & le_mask) - wr.adj;
      const uint32_t b = vb + r;
      const bool on = r < g.rows && ((sm.fw[b >> 5] >> (b & 31u)) & 1u);
      if ((word >> lane) & 1u) {
        n_rows += on ? 1u : 0u;
        continue;
      }
      if (!on) continue;
      const int64_t ei = ebase + (int64_t)xi - (int64_t)r;
      if (ei < 0 || ei >= (int64_t)a.m) {
        a.ctr->error = 1u;
        continue;
      }
      tgt[k] = __ldcs(a.C + ei);
    }
#pragma unroll
    for (int k = 0; k < kWindows; ++k) {
      if (tgt[k] != kNone && tgt[k] >= a.n_rows) {
        a.ctr->error = 1u;
        tgt[k] = kNone;
      }
      const uint32_t tword = tgt[k] == kNone ? kNone : (tgt[k] >> 5);
      const uint32_t tbit = tgt[k] == kNone ? 0u : (1u << (tgt[k] & 31u));
      bool head;
      const uint32_t rm = run_mask(tword, &head);
      const uint32_t bits = __reduce_or_sync(rm, tbit);
      if (head && tword != kNone) atomicOr(a.chg + tword, bits);
      n_edges += tgt[k] != kNone ? 1u : 0u;
    }
    __syncthreads();
    if (tid < kTileWords) sm.isv[tid] = 0u;
    __syncthreads();
  }
  n_rows = __reduce_add_sync(kFull, n_rows);
  n_edges = __reduce_add_sync(kFull, n_edges);
  if (lane == 0) {
    if (n_rows) atomicAdd(&a.ctr->updated, (unsigned long long)n_rows);
    if (n_edges) atomicAdd(&a.ctr->out_edges, (unsigned long long)n_edges);
  }
}

// Dynamic shared memory of the sweep kernels (all static now).
template <typename OffT>
constexpr size_t sweep_smem_bytes() {
  return 0;
}

}  // namespace kites_internal
