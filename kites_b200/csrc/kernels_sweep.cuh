// kernels_sweep.cuh -- the tiled dense sweep over the CSC.
//
// For iterations where most rows (or most sources) are live, walking the
// CSC tile by tile beats per-row discovery.  A tile is kTileItems
// consecutive items of the merged "row, then its in-edges" sequence (row v
// at item v + R[v], its edge e at v + 1 + e).  A CTA first marks the tile's
// vertex items in a shared bitmap (one bit per item) and records each row's
// local position; then each thread takes 8 consecutive items.  An item's row
// is the number of vertex items up to it (prefix popcounts of the bitmap)
// and its edge index follows from the row, so a thread needs no search and
// no walk; it issues the C/E loads and then the V gathers of all 8 items
// back to back.  Row minima fold in registers along the thread's items; the
// first and last row of each thread meet over the warp (runs of equal row)
// and in a shared accumulator; rows that lie wholly in the tile store their
// value, rows split across tiles merge into V with global atomicMin.
//
// Latency: a CTA walks its tiles in sequence, so every dependent round trip
// to memory inside a tile costs the whole CTA.  The next tile's table
// entries and first row offsets are fetched while the current tile works,
// and the old values of the tile's rows are fetched together with its C
// loads; what remains per tile is C -> V.
//
// Modes: kRowFilter -- rows whose frontier bit is set (PLAIN on a dense
// frontier); kAllRows -- every row over every in-edge (PULL_ALL on a dense
// changed set, where testing each source's changed bit would cost one more
// round trip than the gathers it saves; pulling from an unchanged source
// cannot lower a row, so the fixed point is the same).  k_activate_sweep
// computes a dense next frontier by pull over the same tiles.
#pragma once
#include "kernels.cuh"

namespace kites_internal {

constexpr int kSweepThreads = 256;
constexpr int kSweepWarps = kSweepThreads / 32;
constexpr int kTileItems = 2048;                              // items per tile
constexpr int kTileWords = kTileItems / 32;                   // vertex-item bitmap words
constexpr int kRowSlots = kTileItems + 4;                     // rows + 1 <= 2050
constexpr int kFrontierWords = 72;                            // bitmap words of <= 2049 rows
constexpr int kItemsPerThread = kTileItems / kSweepThreads;  // 8
static_assert(32 % kItemsPerThread == 0, "a thread's items share one bitmap word");

enum { kRowFilter = 0, kAllRows = 1 };

template <typename OffT>
struct sweep_args {
  const OffT *R;
  const uint32_t *C;
  const uint32_t *E;
  uint32_t *V;
  const uint32_t *tile_v0;   // chunk table with kTileItems items per chunk
  uint64_t ntiles, n_rows, n_items;
  const uint32_t *rd;        // kRowFilter: frontier bits
  const uint32_t *U;         // k_activate_sweep: the changed set
  uint32_t *chg;             // next changed bits (activation: the frontier written)
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

// A tile's table entries (issued early) and, once they are in, the offset
// R[v0 + threadIdx.x] of the thread's first row (issued before it is used).
template <typename OffT>
struct tile_prefetch {
  uint64_t t;
  uint32_t v0, v1;
  OffT r;
  __device__ __forceinline__ void start(const sweep_args<OffT> &a, uint64_t tile) {
    t = tile;
    v0 = v1 = 0;
    r = 0;
    if (t < a.ntiles) {
      v0 = a.tile_v0[t];
      v1 = a.tile_v0[t + 1];
    }
  }
  __device__ __forceinline__ uint32_t rows(const sweep_args<OffT> &a) const {
    return (uint32_t)(min((uint64_t)v1, a.n_rows - 1) - v0 + 1);
  }
  __device__ __forceinline__ void fetch_r(const sweep_args<OffT> &a) {
    if (t < a.ntiles && threadIdx.x <= rows(a)) r = a.R[(uint64_t)v0 + threadIdx.x];
  }
  __device__ __forceinline__ tile_geom geom(const sweep_args<OffT> &a) const {
    tile_geom g;
    g.item_lo = t * (uint64_t)kTileItems;
    g.nloc = (uint32_t)(min(g.item_lo + (uint64_t)kTileItems, a.n_items) - g.item_lo);
    g.v0 = v0;
    g.rows = rows(a);
    return g;
  }
};

// pos[j] = v0 + j + R[v0 + j] - item_lo for j in [0, rows], clamped to
// [-1, kTileItems + 1] (outside the tile only "before" and "after" matter:
// only row 0 starts before it, only row `rows` after it); the bitmap bit of
// every vertex item inside the tile; acc = `init`; the rows' bitmap words
// from `bits` (when given).  r_first = R[v0 + threadIdx.x] (prefetched).
// isv must be zero on entry.
template <typename OffT>
__device__ __forceinline__ void tile_setup(const sweep_args<OffT> &a, const tile_geom &g,
                                           OffT r_first, const uint32_t *bits, uint32_t init,
                                           sweep_smem &sm) {
  for (uint32_t j = threadIdx.x; j <= g.rows; j += kSweepThreads) {
    const OffT rj = j == threadIdx.x ? r_first : a.R[g.v0 + j];
    const int64_t p = (int64_t)(g.v0 + j) + (int64_t)rj - (int64_t)g.item_lo;
    sm.pos[j] = (int32_t)max((int64_t)-1, min(p, (int64_t)kTileItems + 1));
    if (p >= 0 && p < (int64_t)g.nloc) atomicOr(&sm.isv[p >> 5], 1u << (p & 31));
    if (j < g.rows) sm.acc[j] = init;
  }
  if (bits) {
    const uint32_t nw = ((uint32_t)(g.v0 & 31u) + g.rows + 31u) >> 5;  // <= 66
    for (uint32_t i = threadIdx.x; i < nw; i += kSweepThreads) sm.fw[i] = bits[(g.v0 >> 5) + i];
  }
}

// The thread's items: items 8t .. 8t + 7 of the tile, all inside one bitmap
// word.  The row of an item is the number of vertex items up to and
// including it, minus 1 when the tile starts with row v0's vertex item;
// `before` is that count just ahead of the thread's first item (prefix
// popcounts of the 64 bitmap words, computed by every warp for itself).
// Edge items address C through a per-tile base: edge e = e_first + xi - row
// with e_first = item_lo - v0 - 1, read as base[xi - row - 1] with
// base = item_lo - v0, valid while xi - row - 1 lies in [lo_ok, hi_ok).
struct thread_items {
  uint32_t bits;    // bit k: item k of the thread is a vertex item
  uint32_t before;  // vertex items before the thread's first item, minus adj
  int64_t base;
  int32_t lo_ok, hi_ok;
  __device__ __forceinline__ thread_items(const sweep_smem &sm, const tile_geom &g, uint64_t m) {
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    const uint32_t c0 = __popc(sm.isv[lane]), c1 = __popc(sm.isv[lane + 32]);
    const uint32_t s0 = warp_inclusive_scan(c0), s1 = warp_inclusive_scan(c1);
    const uint32_t t0 = __shfl_sync(kFull, s0, 31);
    const uint32_t ex = w < kSweepWarps / 2 ? s0 - c0 : t0 + s1 - c1;  // warp-uniform choice
    const uint32_t wi = (threadIdx.x * kItemsPerThread) >> 5;         // this thread's word
    const uint32_t sh = (threadIdx.x * kItemsPerThread) & 31u;
    const uint32_t word = sm.isv[wi];
    const uint32_t pfx = __shfl_sync(kFull, ex, wi & 31u);
    bits = (word >> sh) & ((1u << kItemsPerThread) - 1u);
    before = pfx + __popc(word & ((1u << sh) - 1u)) - (sm.pos[0] == 0 ? 1u : 0u);
    base = (int64_t)g.item_lo - (int64_t)g.v0;
    lo_ok = (int32_t)max(-base, (int64_t)INT32_MIN);
    hi_ok = (int32_t)min((int64_t)m - base, (int64_t)INT32_MAX);
  }
};

// Sets the row bits of a warp's 32 consecutive finalised rows (row wv + i
// for lane i when `on`): they share at most two words of `bits`, the second
// touched only when it receives bits.  Returns, in every lane, the bits this
// call set first.
__device__ __forceinline__ uint32_t mark_rows(uint32_t *bits, uint64_t wv, bool on) {
  const uint32_t off = (uint32_t)(wv & 31u);
  const uint32_t bal = __ballot_sync(kFull, on);
  uint32_t fresh = 0;
  if (bal && lane_id() == 0) {
    const uint32_t lo = bal << off, hi = off ? (bal >> (32u - off)) : 0u;
    if (lo) fresh |= (lo & ~atomicOr(bits + (wv >> 5), lo)) >> off;
    if (hi) fresh |= (hi & ~atomicOr(bits + (wv >> 5) + 1, hi)) << (32u - off);
  }
  return __shfl_sync(kFull, fresh, 0);
}

template <int OP, typename OffT, int MODE>
__global__ void __launch_bounds__(kSweepThreads, 4) k_sweep(sweep_args<OffT> a) {
  if (a.ctr->done) return;
  if (a.gate == 2 && !frontier_dense(a.ctr, a.gate_cur, a.dense_edges)) return;
  constexpr bool kW = op_reads_weights<OP>();
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  __shared__ sweep_smem sm;
  const uint32_t tid = threadIdx.x;
  uint32_t n_act = 0, n_edges = 0, n_chg = 0;
  if (tid < kTileWords) sm.isv[tid] = 0u;
  tile_prefetch<OffT> cur, nxt;
  cur.start(a, blockIdx.x);
  cur.fetch_r(a);
  __syncthreads();
  while (cur.t < a.ntiles) {
    const tile_geom g = cur.geom(a);
    tile_setup(a, g, cur.r, MODE == kRowFilter ? a.rd : nullptr, kInf, sm);
    nxt.start(a, cur.t + gridDim.x);
    __syncthreads();
    const thread_items ti(sm, g, a.m);
    const uint32_t vold = tid < g.rows ? a.V[g.v0 + tid] : 0u;  // used when finalising
    const uint32_t vb = (uint32_t)(g.v0 & 31u);
    const uint32_t *Cb = a.C + ti.base;
    const uint32_t *Eb = kW ? a.E + ti.base : nullptr;
    uint32_t row[kItemsPerThread], src[kItemsPerThread], wt[kItemsPerThread];
    int32_t ej[kItemsPerThread];
    {
      uint32_t cnt = ti.before;
#pragma unroll
      for (int k = 0; k < kItemsPerThread; ++k) {
        const uint32_t xi = tid * kItemsPerThread + k;
        const bool vertex = (ti.bits >> k) & 1u;
        cnt += vertex ? 1u : 0u;
        row[k] = xi < g.nloc ? cnt : kNone;
        ej[k] = INT32_MIN;  // no edge to read
        if (xi < g.nloc && !vertex) {
          bool on = true;
          if (MODE == kRowFilter) {
            const uint32_t b = vb + cnt;
            on = (sm.fw[b >> 5] >> (b & 31u)) & 1u;
          }
          const int32_t j = (int32_t)(xi - cnt) - 1;
          if (j < ti.lo_ok || j >= ti.hi_ok || cnt >= g.rows) a.ctr->error = 1u;  // out of step
          else if (on) ej[k] = j;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kItemsPerThread; ++k) {
      const bool live = ej[k] != INT32_MIN;
      src[k] = live ? __ldcs(Cb + ej[k]) : 0u;
      wt[k] = (kW && live) ? __ldcs(Eb + ej[k]) : 0u;
    }
    nxt.fetch_r(a);
    uint32_t cand[kItemsPerThread];
#pragma unroll
    for (int k = 0; k < kItemsPerThread; ++k) {
      bool live = ej[k] != INT32_MIN;
      if (live && src[k] >= a.n_rows) {
        a.ctr->error = 1u;
        live = false;
        ej[k] = INT32_MIN;
      }
      cand[k] = live ? a.V[src[k]] : kInf;
    }
#pragma unroll
    for (int k = 0; k < kItemsPerThread; ++k) {
      const bool live = ej[k] != INT32_MIN;
      cand[k] = live ? nbr_comp<OP>(cand[k], wt[k]) : kInf;
      n_edges += live ? 1u : 0u;
    }
    // Fold into row segments: rows interior to the thread have this thread
    // as their only writer; the first and last segments meet over the warp
    // (runs of equal row) and in shared memory.
    uint32_t seg = kNone, p = kInf, first_row = kNone, first_p = kInf;
    bool first_open = true;
#pragma unroll
    for (int k = 0; k < kItemsPerThread; ++k) {
      if (row[k] == kNone) continue;
      if (row[k] != seg) {
        if (seg != kNone) {
          if (first_open) { first_row = seg; first_p = p; first_open = false; }
          else if (p != kInf) sm.acc[seg] = p;
        }
        seg = row[k];
        p = kInf;
      }
      p = min(p, cand[k]);
    }
    uint32_t fr = seg, fp = p, lr = kNone, lp = kInf;
    if (!first_open) { fr = first_row; fp = first_p; lr = seg; lp = p; }
    {
      bool head;
      const uint32_t rm = run_mask(fr, &head);
      const uint32_t q = __reduce_min_sync(rm, fp);
      if (head && fr != kNone && q != kInf) atomicMin(&sm.acc[fr], q);
    }
    {
      bool head;
      const uint32_t rm = run_mask(lr, &head);
      const uint32_t q = __reduce_min_sync(rm, lp);
      if (head && lr != kNone && q != kInf) atomicMin(&sm.acc[lr], q);
    }
    __syncthreads();
    // Finalise the tile's rows.  A row whose items all lie in the tile has
    // this CTA as its only writer (so its prefetched value is current); a
    // split row merges with atomicMin.
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
          if (whole) {
            const uint32_t old = jb == 0 ? vold : a.V[v];
            if (acc < old) {
              a.V[v] = acc;
              upd = true;
            }
          } else {
            upd = acc < atomicMin(a.V + v, acc);
          }
        }
        if (MODE == kRowFilter) {
          const uint32_t b = vb + j;
          if ((sm.fw[b >> 5] >> (b & 31u)) & 1u)
            n_act += (p0 >= 0 && p0 < (int32_t)g.nloc) ? 1u : 0u;
        }
      }
      const uint32_t fresh = mark_rows(a.chg, g.v0 + jb + (tid & ~31u), upd);
      if (fresh && lane_id() == 0) {
        n_chg += __popc(fresh);
        a.ctr->update_flag = 1u;
      }
    }
    __syncthreads();
    cur = nxt;
  }
  n_act = __reduce_add_sync(kFull, n_act);
  n_edges = __reduce_add_sync(kFull, n_edges);
  n_chg = __reduce_add_sync(kFull, n_chg);
  if (lane_id() == 0) {
    if (n_act) atomicAdd(&a.ctr->active, (unsigned long long)n_act);
    if (n_edges) atomicAdd(&a.ctr->edges, (unsigned long long)n_edges);
    if (n_chg) atomicAdd(&a.ctr->changed, (unsigned long long)n_chg);
  }
}

// Dense activation by pull: vertex v joins the next frontier (chg) iff one
// of its in-edges comes from a vertex of the changed set U -- exactly the
// out-neighbours of U, found over the in-CSC tiles with one load of U per
// in-edge and no atomics per edge (a push expansion pays an atomicOr per
// out-edge of every changed vertex).  Counts: updated += changed rows (bit
// set in U, counted by the tile holding the row's vertex item); out_edges +=
// in-degree of every newly activated row (the edges the next pull reads).
// gate: 2 = run only when the changed set is dense (see expand_args).
template <typename OffT>
__global__ void __launch_bounds__(kSweepThreads, 4) k_activate_sweep(sweep_args<OffT> a) {
  if (a.ctr->done) return;
  if (a.gate == 2 && !changed_dense(a.ctr, a.gate_cur, a.dense_edges)) return;
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  __shared__ sweep_smem sm;
  const uint32_t tid = threadIdx.x, lane = lane_id();
  unsigned long long n_rows = 0, n_edges = 0;
  if (tid < kTileWords) sm.isv[tid] = 0u;
  tile_prefetch<OffT> cur, nxt;
  cur.start(a, blockIdx.x);
  cur.fetch_r(a);
  __syncthreads();
  while (cur.t < a.ntiles) {
    const tile_geom g = cur.geom(a);
    tile_setup(a, g, cur.r, a.U, 1u, sm);  // acc[j] = 1: not reached
    nxt.start(a, cur.t + gridDim.x);
    __syncthreads();
    const thread_items ti(sm, g, a.m);
    const uint32_t *Cb = a.C + ti.base;
    uint32_t row[kItemsPerThread], src[kItemsPerThread];
    uint32_t cnt = ti.before;
#pragma unroll
    for (int k = 0; k < kItemsPerThread; ++k) {
      const uint32_t xi = tid * kItemsPerThread + k;
      const bool vertex = (ti.bits >> k) & 1u;
      cnt += vertex ? 1u : 0u;
      row[k] = kNone;
      src[k] = kNone;
      if (xi >= g.nloc || vertex) continue;
      const int32_t j = (int32_t)(xi - cnt) - 1;
      if (j < ti.lo_ok || j >= ti.hi_ok || cnt >= g.rows) {
        a.ctr->error = 1u;
        continue;
      }
      row[k] = cnt;
      src[k] = __ldcs(Cb + j);
    }
    nxt.fetch_r(a);
    uint32_t uw[kItemsPerThread];
#pragma unroll
    for (int k = 0; k < kItemsPerThread; ++k) {
      if (src[k] != kNone && src[k] >= a.n_rows) {
        a.ctr->error = 1u;
        src[k] = kNone;
        row[k] = kNone;
      }
      uw[k] = src[k] != kNone ? a.U[src[k] >> 5] : 0u;
    }
    // A row is reached if any of its in-edges is: acc[row] = 0.
    uint32_t seg = kNone, hit = 0, first_row = kNone, first_hit = 0;
    bool first_open = true;
#pragma unroll
    for (int k = 0; k < kItemsPerThread; ++k) {
      if (row[k] == kNone) continue;
      if (row[k] != seg) {
        if (seg != kNone) {
          if (first_open) { first_row = seg; first_hit = hit; first_open = false; }
          else if (hit) sm.acc[seg] = 0u;
        }
        seg = row[k];
        hit = 0;
      }
      hit |= (uw[k] >> (src[k] & 31u)) & 1u;
    }
    uint32_t fr = seg, fh = hit, lr = kNone, lh = 0;
    if (!first_open) { fr = first_row; fh = first_hit; lr = seg; lh = hit; }
    {
      bool head;
      const uint32_t rm = run_mask(fr, &head);
      const uint32_t q = __reduce_or_sync(rm, fh);
      if (head && fr != kNone && q) sm.acc[fr] = 0u;
    }
    {
      bool head;
      const uint32_t rm = run_mask(lr, &head);
      const uint32_t q = __reduce_or_sync(rm, lh);
      if (head && lr != kNone && q) sm.acc[lr] = 0u;
    }
    __syncthreads();
    if (tid < kTileWords) sm.isv[tid] = 0u;
    const uint32_t vb = (uint32_t)(g.v0 & 31u);
    for (uint32_t jb = 0; jb < g.rows; jb += kSweepThreads) {
      const uint32_t j = jb + tid;
      bool on = false;
      if (j < g.rows) {
        on = sm.acc[j] == 0u;
        const int32_t p0 = sm.pos[j];
        const uint32_t b = vb + j;
        if (((sm.fw[b >> 5] >> (b & 31u)) & 1u) && p0 >= 0 && p0 < (int32_t)g.nloc) ++n_rows;
      }
      const uint32_t fresh = mark_rows(a.chg, g.v0 + jb + (tid & ~31u), on);
      if ((fresh >> lane) & 1u) {
        const uint64_t v = g.v0 + j;
        n_edges += (unsigned long long)(a.R[v + 1] - a.R[v]);
      }
    }
    __syncthreads();
    cur = nxt;
  }
  n_rows = __reduce_add_sync(kFull, (uint32_t)n_rows);
#pragma unroll
  for (int d = 16; d; d >>= 1) n_edges += __shfl_xor_sync(kFull, n_edges, d);
  if (lane == 0) {
    if (n_rows) atomicAdd(&a.ctr->updated, n_rows);
    if (n_edges) atomicAdd(&a.ctr->out_edges, n_edges);
  }
}

// Dynamic shared memory of the sweep kernels (their shared memory is static).
template <typename OffT>
constexpr size_t sweep_smem_bytes() {
  return 0;
}

}  // namespace kites_internal
