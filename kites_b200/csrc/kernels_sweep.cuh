// kernels_sweep.cuh -- shared-memory-staged dense sweep over the CSC.
//
// For iterations where most rows (or most sources) are live, walking the CSC
// tile by tile beats per-row discovery: a CTA stages a tile of the merged
// "row, then its in-edges" sequence -- the tile's row offsets and the
// contiguous slice of C and E -- into shared memory with 16-byte cp.async
// copies, double-buffered so the next tile streams in while this one is
// reduced.  Each thread then owns kItemsPerThread consecutive items
// (merge-path split, found by a binary search over the staged offsets) and
// issues all of its V[u] gathers back to back.  Row partials meet in a
// shared-memory accumulator: rows interior to a thread store directly,
// rows at thread boundaries are pre-reduced over the warp (runs of equal
// row) and merged with shared atomicMin; rows split across tiles merge
// into V with global atomicMin.
//
// Modes: kRowFilter -- rows whose frontier bit is set (PLAIN on a dense
// frontier); kEdgeFilter -- every row, only in-edges whose source changed
// last iteration (PULL_ALL).
#pragma once
#include "kernels.cuh"

namespace kites_internal {

constexpr int kSweepThreads = 256;
constexpr int kItemsPerThread = 8;
constexpr int kTileItems = kSweepThreads * kItemsPerThread;  // 2048
constexpr int kStageWords = kTileItems + 8;                  // + 16-byte alignment slack

enum { kRowFilter = 0, kEdgeFilter = 1 };

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <typename OffT>
struct sweep_args {
  const OffT *R;
  const uint32_t *C;
  const uint32_t *E;
  uint32_t *V;
  const uint32_t *tile_v0;   // chunk table with kTileItems items per chunk
  uint64_t ntiles, n_rows, n_items;
  const uint32_t *rd;        // kRowFilter: frontier bits
  const uint32_t *U;         // kEdgeFilter: changed bits of the previous iteration
  uint32_t *chg;             // next changed bits (vertex level)
  run_counters *ctr;
  uint64_t m;                // edges (bounds of the staged slices)
  // kRowFilter density gate (see pull_args): 2 = run only on dense frontiers.
  uint32_t gate, gate_cur;
  unsigned long long dense_edges;
};

template <typename OffT>
struct tile_geom {
  uint64_t item_lo, item_hi, v0, v1;  // rows v0..v1 (inclusive)
  uint64_t e_lo, e_hi;                // edges of the tile [e_lo, e_hi)
  uint64_t e_al, r_al;                // 16-byte aligned starts of the staged slices
};

template <typename OffT>
__device__ __forceinline__ tile_geom<OffT> tile_of(const sweep_args<OffT> &a, uint64_t t) {
  tile_geom<OffT> g;
  g.item_lo = t * (uint64_t)kTileItems;
  g.item_hi = min(g.item_lo + (uint64_t)kTileItems, a.n_items);
  g.v0 = a.tile_v0[t];
  g.v1 = a.tile_v0[t + 1];
  if (g.v1 >= a.n_rows) g.v1 = a.n_rows - 1;
  // First edge item at or after item_lo: item_lo itself is in row v0's
  // span.  Edge items before item_hi: item_hi minus the vertex items before
  // it, i.e. rows v0 .. v1 when row v1's vertex item lies inside the tile,
  // else rows v0 .. v1-1 (then the tile ends exactly at R[v1]).
  const int64_t r0 = (int64_t)a.R[g.v0];
  const int64_t rv1 = (int64_t)a.R[g.v1];
  g.e_lo = (uint64_t)max(r0, (int64_t)g.item_lo - (int64_t)g.v0 - 1);
  const bool v1_inside = (uint64_t)((int64_t)g.v1 + rv1) < g.item_hi;
  g.e_hi = v1_inside ? g.item_hi - g.v1 - 1 : (uint64_t)rv1;
  if (g.e_hi < g.e_lo) g.e_hi = g.e_lo;
  const uint64_t per16 = 16 / sizeof(uint32_t);
  g.e_al = g.e_lo & ~(per16 - 1);
  g.r_al = g.v0 & ~(uint64_t)(16 / sizeof(OffT) - 1);
  return g;
}

// Stage R[r_al .. v1+1], C/E[e_al .. e_hi) (rounded up to 16 bytes; the
// pool rounds every allocation to 256 bytes, so the tail stays inside it).
template <typename OffT, bool kWeights>
__device__ __forceinline__ void stage_tile(const sweep_args<OffT> &a, const tile_geom<OffT> &g,
                                           OffT *Rs, uint32_t *Cs, uint32_t *Es) {
  const uint32_t tid = threadIdx.x;
  const uint64_t r_words = (g.v1 + 2 - g.r_al) * sizeof(OffT);        // bytes
  const uint64_t r_chunks = (r_words + 15) / 16;
  for (uint64_t i = tid; i < r_chunks; i += kSweepThreads)
    cp_async16(reinterpret_cast<char *>(Rs) + i * 16,
               reinterpret_cast<const char *>(a.R + g.r_al) + i * 16);
  const uint64_t e_chunks = ((g.e_hi - g.e_al) * 4 + 15) / 16;
  for (uint64_t i = tid; i < e_chunks; i += kSweepThreads) {
    cp_async16(reinterpret_cast<char *>(Cs) + i * 16,
               reinterpret_cast<const char *>(a.C + g.e_al) + i * 16);
    if (kWeights)
      cp_async16(reinterpret_cast<char *>(Es) + i * 16,
                 reinterpret_cast<const char *>(a.E + g.e_al) + i * 16);
  }
}

template <int OP, typename OffT, int MODE>
__global__ void __launch_bounds__(kSweepThreads) k_sweep(sweep_args<OffT> a) {
  if (a.ctr->done) return;
  if (a.gate == 2 && !frontier_dense(a.ctr, a.gate_cur, a.dense_edges)) return;
  constexpr bool kW = op_reads_weights<OP>();
  extern __shared__ __align__(16) unsigned char smem[];
  // Two stage buffers + the row accumulator.
  const uint32_t rwords = (kTileItems + 8) * sizeof(OffT) / 4;
  uint32_t *base = reinterpret_cast<uint32_t *>(smem);
  OffT *Rs[2];
  uint32_t *Cs[2], *Es[2];
  for (int b = 0; b < 2; ++b) {
    uint32_t *p = base + b * (rwords + 2 * kStageWords);
    Rs[b] = reinterpret_cast<OffT *>(p);
    Cs[b] = p + rwords;
    Es[b] = p + rwords + kStageWords;
  }
  uint32_t *acc_s = base + 2 * (rwords + 2 * kStageWords);  // kTileItems + 1 rows
  const uint32_t tid = threadIdx.x, lane = lane_id();
  uint32_t n_act = 0, n_edges = 0, n_chg = 0;
  const uint64_t stride = gridDim.x;
  uint64_t t = blockIdx.x;
  if (t < a.ntiles) stage_tile<OffT, kW>(a, tile_of(a, t), Rs[0], Cs[0], Es[0]);
  cp_async_commit();
  int buf = 0;
  for (; t < a.ntiles; t += stride, buf ^= 1) {
    const tile_geom<OffT> g = tile_of(a, t);
    const uint64_t tn = t + stride;
    if (tn < a.ntiles) stage_tile<OffT, kW>(a, tile_of(a, tn), Rs[buf ^ 1], Cs[buf ^ 1], Es[buf ^ 1]);
    cp_async_commit();
    const uint32_t rows = (uint32_t)(g.v1 - g.v0 + 1);
    for (uint32_t j = tid; j < rows; j += kSweepThreads) acc_s[j] = kInf;
    cp_async_wait<1>();
    __syncthreads();
    const OffT *R_t = Rs[buf] + (g.v0 - g.r_al);          // R_t[j] = R[v0 + j]
    const uint32_t *C_t = Cs[buf] + (g.e_lo - g.e_al);    // C_t[k] = C[e_lo + k]
    const uint32_t *E_t = Es[buf] + (g.e_lo - g.e_al);
    // This thread's items [x0, x1) of the merged sequence.
    const uint64_t x0 = g.item_lo + (uint64_t)tid * kItemsPerThread;
    const uint64_t x1 = min(x0 + (uint64_t)kItemsPerThread, g.item_hi);
    uint32_t row = 0;  // local row holding item x0: largest j with v0+j+R[v0+j] <= x0
    if (x0 < x1) {
      uint32_t lo = 0, hi = rows;  // answer in [0, rows)
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (g.v0 + mid + (uint64_t)R_t[mid] <= x0) lo = mid; else hi = mid;
      }
      row = lo;
    }
    // Walk the items; segments are (row, partial min).
    uint32_t seg_row = row, first_row = row, p = kInf, first_p = kInf;
    bool first_open = true, row_on = false;
    auto row_active = [&](uint32_t j) -> bool {
      if (MODE == kEdgeFilter) return true;
      const uint64_t v = g.v0 + j;
      return (a.rd[v >> 5] >> (v & 31u)) & 1u;
    };
    uint32_t cand[kItemsPerThread];
    uint32_t crow[kItemsPerThread];
#pragma unroll
    for (int k = 0; k < kItemsPerThread; ++k) { cand[k] = kInf; crow[k] = 0xFFFFFFFFu; }
    // Pass 1: issue every gather (independent loads in flight).
    {
      uint32_t r = row;
      row_on = (x0 < x1) && row_active(r);
#pragma unroll
      for (int k = 0; k < kItemsPerThread; ++k) {
        const uint64_t x = x0 + k;
        if (x >= x1) break;
        if (r + 1 < rows + 1 && g.v0 + r + 1 + (uint64_t)R_t[r + 1] == x) {
          ++r;  // vertex item of row r
          row_on = row_active(r);
          continue;
        }
        if (x == g.v0 + r + (uint64_t)R_t[r]) continue;  // the start row's own vertex item
        const uint64_t e = x - (g.v0 + r) - 1;  // global edge index
        crow[k] = r;
        if (!row_on) continue;
        const uint32_t u = C_t[e - g.e_lo];
        if (u >= a.n_rows || e >= g.e_hi) {  // staged slice out of step: never gather
          a.ctr->error = 1u;
          continue;
        }
        if (MODE == kEdgeFilter && !((a.U[u >> 5] >> (u & 31u)) & 1u)) continue;
        const uint32_t w = kW ? E_t[e - g.e_lo] : 0u;
        cand[k] = nbr_comp<OP>(a.V[u], w);
        ++n_edges;
      }
    }
    // Pass 2: fold candidates into row segments.
    {
#pragma unroll
      for (int k = 0; k < kItemsPerThread; ++k) {
        if (crow[k] == 0xFFFFFFFFu) continue;
        if (crow[k] != seg_row) {
          if (first_open) { first_p = p; first_row = seg_row; first_open = false; }
          else if (p != kInf) acc_s[seg_row] = p;  // interior row: only writer
          seg_row = crow[k];
          p = kInf;
        }
        p = min(p, cand[k]);
      }
    }
    // Thread-boundary segments: first (and last, if different) via warp runs.
    uint32_t fr = 0xFFFFFFFFu, fp = kInf, lr = 0xFFFFFFFFu, lp = kInf;
    if (x0 < x1) {
      if (first_open) { fr = seg_row; fp = p; }
      else { fr = first_row; fp = first_p; lr = seg_row; lp = p; }
    }
    {
      bool head;
      const uint32_t rm = run_mask(fr, &head);
      const uint32_t q = __reduce_min_sync(rm, fp);
      if (head && fr != 0xFFFFFFFFu && q != kInf) atomicMin(acc_s + fr, q);
    }
    {
      bool head;
      const uint32_t rm = run_mask(lr, &head);
      const uint32_t q = __reduce_min_sync(rm, lp);
      if (head && lr != 0xFFFFFFFFu && q != kInf) atomicMin(acc_s + lr, q);
    }
    __syncthreads();
    // Finalise the tile's rows.
    for (uint32_t jb = 0; jb < rows; jb += kSweepThreads) {
      const uint32_t j = jb + tid;
      bool upd = false;
      uint64_t v = g.v0 + j;
      if (j < rows) {
        const uint32_t acc = acc_s[j];
        if (acc != kInf) {
          const int64_t r0 = (int64_t)R_t[j], r1 = (int64_t)R_t[j + 1];
          const bool whole = (int64_t)g.item_lo <= (int64_t)v + r0 &&
                             (int64_t)v + r1 < (int64_t)g.item_hi;
          const uint32_t old = a.V[v];
          if (acc < old) upd = whole ? (a.V[v] = acc, true) : (acc < atomicMin(a.V + v, acc));
        }
      }
      // Vertices of 32 consecutive rows share at most two words; the second
      // word is touched only when it receives bits (of vertices < n).
      const uint32_t bit = upd ? 1u : 0u;
      const uint64_t w0 = (g.v0 + jb + (tid & ~31u)) >> 5;
      const uint32_t off = (uint32_t)((g.v0 + jb + (tid & ~31u)) & 31u);
      const uint32_t bal = __ballot_sync(kFull, bit);
      if (bal && lane == 0) {
        const uint32_t lo = bal << off, hi = off ? (bal >> (32u - off)) : 0u;
        if (lo) n_chg += __popc(lo & ~atomicOr(a.chg + w0, lo));
        if (hi) n_chg += __popc(hi & ~atomicOr(a.chg + w0 + 1, hi));
        a.ctr->update_flag = 1u;
      }
      if (j < rows && MODE == kRowFilter && row_active(j)) {
        const int64_t vp = (int64_t)v + (int64_t)R_t[j];
        n_act += (vp >= (int64_t)g.item_lo && vp < (int64_t)g.item_hi) ? 1u : 0u;
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  n_act = __reduce_add_sync(kFull, n_act);
  n_edges = __reduce_add_sync(kFull, n_edges);
  n_chg = __reduce_add_sync(kFull, n_chg);
  if (lane == 0) {
    if (n_act) atomicAdd(&a.ctr->active, (unsigned long long)n_act);
    if (n_edges) atomicAdd(&a.ctr->edges, (unsigned long long)n_edges);
    if (n_chg) atomicAdd(&a.ctr->changed, (unsigned long long)n_chg);
  }
}

// Dense activation: the same staged tiles over the activation adjacency
// (rows = changed candidates, C = targets); every edge of a row whose bit is
// set in chg ORs its target's bit into wr.  gate: 2 = run only when the
// activation is dense (see pull_args), 1 = only when sparse, 0 = always.
template <typename OffT>
__global__ void __launch_bounds__(kSweepThreads) k_expand_sweep(sweep_args<OffT> a) {
  if (a.ctr->done) return;
  if (a.gate == 2 && !changed_dense(a.ctr, a.gate_cur, a.dense_edges)) return;
  // Here rd = the changed rows, chg = the frontier being written.
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t rwords = (kTileItems + 8) * sizeof(OffT) / 4;
  uint32_t *base = reinterpret_cast<uint32_t *>(smem);
  OffT *Rs[2];
  uint32_t *Cs[2];
  for (int b = 0; b < 2; ++b) {
    uint32_t *p = base + b * (rwords + 2 * kStageWords);
    Rs[b] = reinterpret_cast<OffT *>(p);
    Cs[b] = p + rwords;
  }
  const uint32_t tid = threadIdx.x, lane = lane_id();
  uint32_t n_rows = 0, n_edges = 0;
  const uint64_t stride = gridDim.x;
  uint64_t t = blockIdx.x;
  if (t < a.ntiles) stage_tile<OffT, false>(a, tile_of(a, t), Rs[0], Cs[0], nullptr);
  cp_async_commit();
  int buf = 0;
  for (; t < a.ntiles; t += stride, buf ^= 1) {
    const tile_geom<OffT> g = tile_of(a, t);
    const uint64_t tn = t + stride;
    if (tn < a.ntiles) stage_tile<OffT, false>(a, tile_of(a, tn), Rs[buf ^ 1], Cs[buf ^ 1], nullptr);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const uint32_t rows = (uint32_t)(g.v1 - g.v0 + 1);
    const OffT *R_t = Rs[buf] + (g.v0 - g.r_al);
    const uint32_t *C_t = Cs[buf] + (g.e_lo - g.e_al);
    const uint64_t x0 = g.item_lo + (uint64_t)tid * kItemsPerThread;
    const uint64_t x1 = min(x0 + (uint64_t)kItemsPerThread, g.item_hi);
    if (x0 < x1) {
      uint32_t lo = 0, hi = rows;
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (g.v0 + mid + (uint64_t)R_t[mid] <= x0) lo = mid; else hi = mid;
      }
      uint32_t r = lo;
      bool on = (a.rd[(g.v0 + r) >> 5] >> ((g.v0 + r) & 31u)) & 1u;
#pragma unroll
      for (int k = 0; k < kItemsPerThread; ++k) {
        const uint64_t x = x0 + k;
        if (x >= x1) break;
        if (r + 1 <= rows && g.v0 + r + 1 + (uint64_t)R_t[r + 1] == x) {
          ++r;
          const uint64_t v = g.v0 + r;
          on = (a.rd[v >> 5] >> (v & 31u)) & 1u;
          n_rows += on ? 1u : 0u;
          continue;
        }
        if (x == g.v0 + r + (uint64_t)R_t[r]) {  // the start row's own vertex item
          n_rows += on ? 1u : 0u;
          continue;
        }
        if (!on) continue;
        const uint64_t e = x - (g.v0 + r) - 1;
        const uint32_t tgt = C_t[e - g.e_lo];
        if (tgt >= a.n_rows || e >= g.e_hi) {  // staged slice out of step
          a.ctr->error = 1u;
          continue;
        }
        atomicOr(a.chg + (tgt >> 5), 1u << (tgt & 31u));
        ++n_edges;
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  n_rows = __reduce_add_sync(kFull, n_rows);
  n_edges = __reduce_add_sync(kFull, n_edges);
  if (lane == 0) {
    if (n_rows) atomicAdd(&a.ctr->updated, (unsigned long long)n_rows);
    if (n_edges) atomicAdd(&a.ctr->out_edges, (unsigned long long)n_edges);
  }
}

template <typename OffT>
constexpr size_t sweep_smem_bytes() {
  return (size_t)2 * ((kTileItems + 8) * sizeof(OffT) + 2 * kStageWords * 4) +
         (size_t)(kTileItems + 1) * 4;
}

}  // namespace kites_internal
