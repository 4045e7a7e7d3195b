// kernels_sweep.cuh -- the dense sweep: edge-parallel passes over the CSC.
//
// For iterations where most rows (or most sources) are live, every in-edge
// is read anyway, so the work is laid out by edge, not by row: each thread
// takes 8 consecutive edges (two 16-byte loads each of C, E and the per-edge
// row index `rowid`, built once at upload), all of its V gathers are in
// flight together, and the rows' minima fold in registers along the
// thread's edges (rows are sorted, so a row is a run of equal `rowid`).  A
// row lying inside one thread's 8 edges is finished by that thread; the
// first and last row of a thread meet their neighbours over the warp (runs
// of equal row, `__reduce_min_sync`); whatever crosses a warp's 256-edge
// window merges into V with atomicMin.  A row is written only when its
// minimum beats the value read before the fold, and atomicMin's return says
// whether this warp lowered it (the changed bit).  The row index costs 4
// bytes per edge more than the item-merged walk it replaces and saves
// almost all of its per-item arithmetic.
//
// Modes: kRowFilter -- rows whose frontier bit is set (PLAIN on a dense
// frontier; V gathers are issued with the frontier words, so edges of
// inactive rows cost a gather but no extra round trip); kAllRows -- every
// row over every in-edge (PULL_ALL on a dense changed set; pulling from an
// unchanged source cannot lower a row, so the fixed point is the same).
// k_activate_sweep computes a dense next frontier by pull with the same
// layout.
#pragma once
#include "kernels.cuh"

namespace kites_internal {

constexpr int kSweepThreads = 256;
constexpr int kEdgesPerThread = 8;
constexpr int kWindowEdges = 32 * kEdgesPerThread;  // edges per warp step
// Five CTAs (40 warps) per SM: more gathers in flight than four at 64
// registers (measured 3 % faster at R-MAT scale 24; six or eight CTAs spill
// and run slower).
constexpr int kSweepMinBlocks = 5;

enum { kRowFilter = 0, kAllRows = 1 };

template <typename OffT>
struct sweep_args {
  const OffT *R;
  const uint32_t *C;
  const uint32_t *E;
  const uint32_t *rowid;     // row of every edge
  uint32_t *V;
  uint64_t m, n_rows;
  const uint32_t *rd;        // kRowFilter: frontier bits
  const uint32_t *U;         // k_activate_sweep: the changed set
  uint32_t *chg;             // next changed bits (activation: the frontier written)
  run_counters *ctr;
  // Density gate (see pull_args / expand_args): 2 = run only when dense.
  uint32_t gate, gate_cur;
  unsigned long long dense_edges;
  uint32_t *act;             // k_sweep_changed: the rows found active
};

constexpr uint32_t kNoRow = 0xFFFFFFFFu;

// Loads the thread's 8 edges starting at e0 (a multiple of 8): whole 16-byte
// vectors when they all exist, element by element at the tail (row = kNoRow
// past m).  `x` receives the rows, `y` the values of `col`.
__device__ __forceinline__ void load_edges8(const uint32_t *__restrict__ rowid,
                                            const uint32_t *__restrict__ col, uint64_t e0,
                                            uint64_t m, uint32_t (&x)[kEdgesPerThread],
                                            uint32_t (&y)[kEdgesPerThread]) {
  if (e0 + kEdgesPerThread <= m) {
    const uint4 r0 = __ldcs(reinterpret_cast<const uint4 *>(rowid + e0));
    const uint4 r1 = __ldcs(reinterpret_cast<const uint4 *>(rowid + e0 + 4));
    const uint4 c0 = __ldcs(reinterpret_cast<const uint4 *>(col + e0));
    const uint4 c1 = __ldcs(reinterpret_cast<const uint4 *>(col + e0 + 4));
    x[0] = r0.x; x[1] = r0.y; x[2] = r0.z; x[3] = r0.w;
    x[4] = r1.x; x[5] = r1.y; x[6] = r1.z; x[7] = r1.w;
    y[0] = c0.x; y[1] = c0.y; y[2] = c0.z; y[3] = c0.w;
    y[4] = c1.x; y[5] = c1.y; y[6] = c1.z; y[7] = c1.w;
  } else {
#pragma unroll
    for (int k = 0; k < kEdgesPerThread; ++k) {
      const bool in = e0 + k < m;
      x[k] = in ? rowid[e0 + k] : kNoRow;
      y[k] = in ? col[e0 + k] : 0u;
    }
  }
}

__device__ __forceinline__ void load_vals8(const uint32_t *__restrict__ p, uint64_t e0, uint64_t m,
                                           uint32_t (&y)[kEdgesPerThread]) {
  if (e0 + kEdgesPerThread <= m) {
    const uint4 a = __ldcs(reinterpret_cast<const uint4 *>(p + e0));
    const uint4 b = __ldcs(reinterpret_cast<const uint4 *>(p + e0 + 4));
    y[0] = a.x; y[1] = a.y; y[2] = a.z; y[3] = a.w;
    y[4] = b.x; y[5] = b.y; y[6] = b.z; y[7] = b.w;
  } else {
#pragma unroll
    for (int k = 0; k < kEdgesPerThread; ++k) y[k] = e0 + k < m ? p[e0 + k] : 0u;
  }
}

template <int OP, typename OffT, int MODE>
__global__ void __launch_bounds__(kSweepThreads, kSweepMinBlocks) k_sweep(sweep_args<OffT> a) {
  if (a.ctr->done) return;
  if (a.gate == 2 && !frontier_dense(a.ctr, a.gate_cur, a.dense_edges)) return;
  constexpr bool kW = op_reads_weights<OP>();
  const uint32_t lane = lane_id();
  uint32_t n_act = 0, n_edges = 0, n_chg = 0;
  bool any_upd = false;
  const uint64_t warps = (uint64_t)gridDim.x * (kSweepThreads / 32);
  for (uint64_t win = ((uint64_t)blockIdx.x * kSweepThreads + threadIdx.x) >> 5;
       win * kWindowEdges < a.m; win += warps) {
    const uint64_t e0 = win * kWindowEdges + (uint64_t)lane * kEdgesPerThread;
    uint32_t row[kEdgesPerThread], src[kEdgesPerThread], wt[kEdgesPerThread];
    load_edges8(a.rowid, a.C, e0, a.m, row, src);
    if (kW) load_vals8(a.E, e0, a.m, wt);
    // The row just before the thread's first edge (to spot row starts).
    uint32_t prev = __shfl_up_sync(kFull, row[kEdgesPerThread - 1], 1);
    if (lane == 0) prev = e0 > 0 && e0 <= a.m ? a.rowid[e0 - 1] : kNoRow;
    // Every window but the last has all of its 8 edges per thread: the fast
    // path below needs no per-edge validity tests and folds branch-free.
    if (__all_sync(kFull, e0 + kEdgesPerThread <= a.m)) {
      uint32_t mx = 0;
#pragma unroll
      for (int k = 0; k < kEdgesPerThread; ++k) mx = max(mx, max(row[k], src[k]));
      const bool bad = mx >= a.n_rows || row[0] > row[kEdgesPerThread - 1];
      if (bad) raise_error(a.ctr, kErrIndex);  // never index with an id out of range
      uint32_t val[kEdgesPerThread], fw[kEdgesPerThread];
      uint32_t w_first = kFull, w_last = kFull;
      if (MODE == kRowFilter && !bad) {
        w_first = a.rd[row[0] >> 5];
        w_last = a.rd[row[kEdgesPerThread - 1] >> 5];
      }
#pragma unroll
      for (int k = 0; k < kEdgesPerThread; ++k) {
        val[k] = bad ? kInf : a.V[src[k]];
        if (MODE == kRowFilter) {
          const uint32_t wd = row[k] >> 5;
          fw[k] = bad ? 0u
                      : wd == (row[0] >> 5) ? w_first
                      : wd == (row[kEdgesPerThread - 1] >> 5) ? w_last
                                                               : a.rd[wd];
        } else {
          fw[k] = bad ? 0u : kFull;
        }
      }
      const uint32_t r0 = bad ? kNoRow : row[0];
      const uint32_t r7 = bad ? kNoRow : row[kEdgesPerThread - 1];
      const uint32_t old_first = bad ? 0u : a.V[r0];
      const uint32_t old_last = bad ? 0u : a.V[r7];
      uint32_t cand[kEdgesPerThread];
#pragma unroll
      for (int k = 0; k < kEdgesPerThread; ++k) {
        const bool on = (fw[k] >> (row[k] & 31u)) & 1u;
        cand[k] = on ? nbr_comp<OP>(val[k], wt[k]) : kInf;
        n_edges += on ? 1u : 0u;
        // Active rows (row starts in this window), counted in both modes: the
        // selector's features read them.
        n_act += (on && row[k] != (k ? row[k - 1] : prev)) ? 1u : 0u;
      }
      // Runs of equal row: p is the running minimum of the current run.
      uint32_t p = cand[0], fp = kInf;
#pragma unroll
      for (int k = 1; k < kEdgesPerThread; ++k) {
        const bool same = row[k] == row[k - 1];
        if (!same && !bad) {
          if (row[k - 1] == r0) {
            fp = p;  // the first run ends
          } else if (p != kInf) {  // a row wholly inside this thread
            const uint32_t sr = row[k - 1];
            if (p < atomicMin(a.V + sr, p)) {
              any_upd = true;
              n_chg += __popc((1u << (sr & 31u)) & ~atomicOr(a.chg + (sr >> 5), 1u << (sr & 31u)));
            }
          }
        }
        p = same ? min(p, cand[k]) : cand[k];
      }
      uint32_t lr = kNoRow, lp = kInf;
      if (r7 == r0) fp = p;
      else { lr = r7; lp = p; }
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const uint32_t r = side ? lr : r0;
        const uint32_t v = side ? lp : fp;
        const uint32_t o = side ? old_last : old_first;
        bool head;
        const uint32_t rm = run_mask(r, &head);
        const uint32_t q = __reduce_min_sync(rm, v);
        if (head && r != kNoRow && q < o) {
          const uint32_t got = atomicMin(a.V + r, q);
          if (q < got) {
            any_upd = true;
            n_chg += __popc((1u << (r & 31u)) & ~atomicOr(a.chg + (r >> 5), 1u << (r & 31u)));
          }
        }
      }
      continue;
    }
    // The last window: edges past m (row kNoRow) and every test per edge.
    // Gathers: V[src] of every edge, the frontier words (row filter), and
    // the current values of the thread's first and last rows.
    uint32_t val[kEdgesPerThread], fw[kEdgesPerThread];
    bool live[kEdgesPerThread];
#pragma unroll
    for (int k = 0; k < kEdgesPerThread; ++k) {
      live[k] = row[k] != kNoRow;
      if (live[k] && (src[k] >= a.n_rows || row[k] >= a.n_rows)) {
        raise_error(a.ctr, kErrIndex);  // never index with an id out of range
        live[k] = false;
        row[k] = kNoRow;
      }
      val[k] = live[k] ? a.V[src[k]] : kInf;
      fw[k] = (MODE == kRowFilter && live[k]) ? a.rd[row[k] >> 5] : kFull;
    }
    uint32_t r_first = kNoRow, r_last = kNoRow;  // the thread's first and last valid rows
#pragma unroll
    for (int k = kEdgesPerThread - 1; k >= 0; --k)
      if (row[k] != kNoRow) r_first = row[k];
#pragma unroll
    for (int k = 0; k < kEdgesPerThread; ++k)
      if (row[k] != kNoRow) r_last = row[k];
    const uint32_t old_first = r_first != kNoRow ? a.V[r_first] : 0u;
    const uint32_t old_last = r_last != kNoRow ? a.V[r_last] : 0u;
    // Fold along the thread's edges; count row starts of active rows.
    uint32_t seg = kNoRow, p = kInf, first_row = kNoRow, first_p = kInf;
    bool first_open = true;
    uint32_t before = prev;
#pragma unroll
    for (int k = 0; k < kEdgesPerThread; ++k) {
      const bool on = live[k] && ((fw[k] >> (row[k] & 31u)) & 1u);
      if (live[k] && row[k] != before && on) ++n_act;
      before = row[k];
      const uint32_t cand = on ? nbr_comp<OP>(val[k], wt[k]) : kInf;
      n_edges += on ? 1u : 0u;
      if (row[k] == kNoRow) continue;
      if (row[k] != seg) {
        if (seg != kNoRow) {
          if (first_open) {
            first_row = seg;
            first_p = p;
            first_open = false;
          } else if (p != kInf) {  // a row wholly inside this thread
            const uint32_t o = atomicMin(a.V + seg, p);
            if (p < o) {
              any_upd = true;
              n_chg += __popc((1u << (seg & 31u)) & ~atomicOr(a.chg + (seg >> 5), 1u << (seg & 31u)));
            }
          }
        }
        seg = row[k];
        p = kInf;
      }
      p = min(p, cand);
    }
    // fr/lr: the thread's first and last rows (r_first / r_last) with their
    // partial minima; one row only: fr alone.
    uint32_t fr = seg, fp = p, lr = kNoRow, lp = kInf;
    if (!first_open) {
      fr = first_row;
      fp = first_p;
      lr = seg;
      lp = p;
    }
    const uint32_t fold = old_first, lold = old_last;
    // First and last rows of each thread, merged over the warp.
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const uint32_t r = side ? lr : fr;
      const uint32_t v = side ? lp : fp;
      const uint32_t o = side ? lold : fold;
      bool head;
      const uint32_t rm = run_mask(r, &head);
      const uint32_t q = __reduce_min_sync(rm, v);
      if (head && r != kNoRow && q < o) {
        const uint32_t got = atomicMin(a.V + r, q);
        if (q < got) {
          any_upd = true;
          n_chg += __popc((1u << (r & 31u)) & ~atomicOr(a.chg + (r >> 5), 1u << (r & 31u)));
        }
      }
    }
  }
  if (__any_sync(kFull, any_upd) && lane == 0) a.ctr->update_flag = 1u;
  n_act = __reduce_add_sync(kFull, n_act);
  n_edges = __reduce_add_sync(kFull, n_edges);
  n_chg = __reduce_add_sync(kFull, n_chg);
  if (lane == 0) {
    if (n_act) atomicAdd(&a.ctr->active, (unsigned long long)n_act);
    if (n_edges) atomicAdd(&a.ctr->edges, (unsigned long long)n_edges);
    if (n_chg) atomicAdd(&a.ctr->changed, (unsigned long long)n_chg);
  }
}

// PLAIN over a dense changed set without a materialised frontier (the
// activation of the previous iteration and this pull in one pass).  Row v
// is active iff one of its in-edges comes from a vertex of U, the previous
// iteration's changed set -- exactly the rows the activation would have
// set -- and only those in-edges are folded: an in-edge from a source that
// did not change was folded when that source last changed (the change
// activated v for the iteration after it), so it cannot lower v, and the
// fixed point and the per-iteration work are the plain strategy's.  The V
// gather of an edge is issued only when its source changed.  Counts as the
// plain pull: a row's activity bit goes into `act` with atomicOr, and the
// thread that sets it counts the row and its in-degree.
// Gate: run only when U has more than dense_edges rows (here the changed-row
// threshold), read from the counters of the previous iteration.
template <int OP, typename OffT>
__global__ void __launch_bounds__(kSweepThreads, kSweepMinBlocks)
    k_sweep_changed(sweep_args<OffT> a) {
  if (a.ctr->done) return;
  if (!changed_dense(a.ctr, a.gate_cur, a.dense_edges)) return;
  constexpr bool kW = op_reads_weights<OP>();
  const uint32_t lane = lane_id();
  unsigned long long n_act = 0, n_edges = 0;
  uint32_t n_chg = 0;
  bool any_upd = false;
  auto mark = [&](uint32_t r) {
    const uint32_t bit = 1u << (r & 31u);
    if (bit & ~atomicOr(a.act + (r >> 5), bit)) {
      ++n_act;
      n_edges += (unsigned long long)(a.R[r + 1] - a.R[r]);
    }
  };
  auto lower = [&](uint32_t r, uint32_t q) {
    if (q < atomicMin(a.V + r, q)) {
      any_upd = true;
      n_chg += __popc((1u << (r & 31u)) & ~atomicOr(a.chg + (r >> 5), 1u << (r & 31u)));
    }
  };
  const uint64_t warps = (uint64_t)gridDim.x * (kSweepThreads / 32);
  for (uint64_t win = ((uint64_t)blockIdx.x * kSweepThreads + threadIdx.x) >> 5;
       win * kWindowEdges < a.m; win += warps) {
    const uint64_t e0 = win * kWindowEdges + (uint64_t)lane * kEdgesPerThread;
    uint32_t row[kEdgesPerThread], src[kEdgesPerThread], wt[kEdgesPerThread];
    load_edges8(a.rowid, a.C, e0, a.m, row, src);
    if (kW) load_vals8(a.E, e0, a.m, wt);
    if (__all_sync(kFull, e0 + kEdgesPerThread <= a.m)) {
      uint32_t mx = 0;
#pragma unroll
      for (int k = 0; k < kEdgesPerThread; ++k) mx = max(mx, max(row[k], src[k]));
      const bool bad = mx >= a.n_rows || row[0] > row[kEdgesPerThread - 1];
      if (bad) raise_error(a.ctr, kErrIndex);  // never index with an id out of range
      // V is gathered only for sources in U.  Loading it for every edge
      // together with the U words (one round trip instead of two dependent
      // ones) was measured slower: 882.7 against 725.8 ms per 64 sources at
      // R-MAT scale 24, the dense sweeps at 0.36 against 0.48 of the copy
      // peak -- the extra gathers cost more than the saved latency.  So was
      // one gather per edge from an array holding V on U and kInf elsewhere,
      // written before the sweep: 832.2 against 728.7 ms, with 7 % more
      // iterations (that copy of V misses the values lowered earlier in the
      // same iteration, which the live V read passes on at once).
      uint32_t hit[kEdgesPerThread], cand[kEdgesPerThread];
#pragma unroll
      for (int k = 0; k < kEdgesPerThread; ++k) {
        const uint32_t uw = bad ? 0u : a.U[src[k] >> 5];
        hit[k] = (uw >> (src[k] & 31u)) & 1u;
      }
#pragma unroll
      for (int k = 0; k < kEdgesPerThread; ++k)
        cand[k] = hit[k] ? nbr_comp<OP>(a.V[src[k]], wt[k]) : kInf;
      const uint32_t r0 = bad ? kNoRow : row[0];
      const uint32_t r7 = bad ? kNoRow : row[kEdgesPerThread - 1];
      const uint32_t old_first = bad ? 0u : a.V[r0];
      const uint32_t old_last = bad ? 0u : a.V[r7];
      // Runs of equal row: p the running minimum, h whether a source changed.
      uint32_t p = cand[0], fp = kInf, h = hit[0], fh = 0;
#pragma unroll
      for (int k = 1; k < kEdgesPerThread; ++k) {
        const bool same = row[k] == row[k - 1];
        if (!same && !bad) {
          if (row[k - 1] == r0) {
            fp = p;  // the first run ends
            fh = h;
          } else if (h) {  // a row wholly inside this thread
            mark(row[k - 1]);
            if (p != kInf) lower(row[k - 1], p);
          }
        }
        p = same ? min(p, cand[k]) : cand[k];
        h = same ? (h | hit[k]) : hit[k];
      }
      uint32_t lr = kNoRow, lp = kInf, lh = 0;
      if (r7 == r0) { fp = p; fh = h; }
      else { lr = r7; lp = p; lh = h; }
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const uint32_t r = side ? lr : r0;
        bool head;
        const uint32_t rm = run_mask(r, &head);
        const uint32_t q = __reduce_min_sync(rm, side ? lp : fp);
        const uint32_t qh = __reduce_or_sync(rm, side ? lh : fh);
        if (head && r != kNoRow && qh) {
          mark(r);
          if (q < (side ? old_last : old_first)) lower(r, q);
        }
      }
      continue;
    }
    // The last window: edge by edge (at most 256 edges per launch).
#pragma unroll
    for (int k = 0; k < kEdgesPerThread; ++k) {
      if (row[k] == kNoRow) continue;
      if (src[k] >= a.n_rows || row[k] >= a.n_rows) {
        raise_error(a.ctr, kErrIndex);  // never index with an id out of range
        continue;
      }
      if (!((a.U[src[k] >> 5] >> (src[k] & 31u)) & 1u)) continue;
      mark(row[k]);
      const uint32_t c = nbr_comp<OP>(a.V[src[k]], wt[k]);
      if (c < a.V[row[k]]) lower(row[k], c);
    }
  }
  if (__any_sync(kFull, any_upd) && lane == 0) a.ctr->update_flag = 1u;
  n_chg = __reduce_add_sync(kFull, n_chg);
#pragma unroll
  for (int d = 16; d; d >>= 1) {
    n_act += __shfl_xor_sync(kFull, n_act, d);
    n_edges += __shfl_xor_sync(kFull, n_edges, d);
  }
  if (lane == 0) {
    if (n_act) atomicAdd(&a.ctr->active, n_act);
    if (n_edges) atomicAdd(&a.ctr->edges, n_edges);
    if (n_chg) atomicAdd(&a.ctr->changed, (unsigned long long)n_chg);
  }
}

// Dense activation by pull: vertex v joins the next frontier (chg) iff one
// of its in-edges comes from a vertex of the changed set U -- exactly the
// out-neighbours of U -- with one load of U per in-edge and an atomicOr per
// activated row (a push expansion pays an atomicOr per out-edge of every
// changed vertex).  Counts: updated += changed rows that have in-edges (the
// thread holding the row's first edge counts it); out_edges += in-degree of
// every newly activated row (the edges the next pull reads).
// gate: 2 = run only when the changed set is dense (see expand_args).
template <typename OffT>
__global__ void __launch_bounds__(kSweepThreads) k_activate_sweep(sweep_args<OffT> a) {
  if (a.ctr->done) return;
  if (a.gate == 2 && !changed_dense(a.ctr, a.gate_cur, a.dense_edges)) return;
  const uint32_t lane = lane_id();
  unsigned long long n_rows = 0, n_edges = 0;
  const uint64_t warps = (uint64_t)gridDim.x * (kSweepThreads / 32);
  for (uint64_t win = ((uint64_t)blockIdx.x * kSweepThreads + threadIdx.x) >> 5;
       win * kWindowEdges < a.m; win += warps) {
    const uint64_t e0 = win * kWindowEdges + (uint64_t)lane * kEdgesPerThread;
    uint32_t row[kEdgesPerThread], src[kEdgesPerThread];
    load_edges8(a.rowid, a.C, e0, a.m, row, src);
    uint32_t prev = __shfl_up_sync(kFull, row[kEdgesPerThread - 1], 1);
    if (lane == 0) prev = e0 > 0 && e0 <= a.m ? a.rowid[e0 - 1] : kNoRow;
    auto activate = [&](uint32_t r) {
      const uint32_t bit = 1u << (r & 31u);
      if (bit & ~atomicOr(a.chg + (r >> 5), bit))
        n_edges += (unsigned long long)(a.R[r + 1] - a.R[r]);
    };
    // Full windows (all but the last): no per-edge validity tests, runs of
    // equal row folded with selects.
    if (__all_sync(kFull, e0 + kEdgesPerThread <= a.m)) {
      uint32_t mx = 0;
#pragma unroll
      for (int k = 0; k < kEdgesPerThread; ++k) mx = max(mx, max(row[k], src[k]));
      const bool bad = mx >= a.n_rows || row[0] > row[kEdgesPerThread - 1];
      if (bad) raise_error(a.ctr, kErrIndex);
      uint32_t hit[kEdgesPerThread];
#pragma unroll
      for (int k = 0; k < kEdgesPerThread; ++k) {
        const uint32_t uw = bad ? 0u : a.U[src[k] >> 5];
        hit[k] = (uw >> (src[k] & 31u)) & 1u;
        // The row's own changed bit, read at row starts only.
        const bool start = !bad && row[k] != (k ? row[k - 1] : prev);
        const uint32_t rw = start ? a.U[row[k] >> 5] : 0u;
        n_rows += (rw >> (row[k] & 31u)) & 1u;
      }
      const uint32_t r0 = bad ? kNoRow : row[0];
      const uint32_t r7 = bad ? kNoRow : row[kEdgesPerThread - 1];
      uint32_t h = hit[0], fh = 0;
#pragma unroll
      for (int k = 1; k < kEdgesPerThread; ++k) {
        const bool same = row[k] == row[k - 1];
        if (!same && !bad) {
          if (row[k - 1] == r0) fh = h;
          else if (h) activate(row[k - 1]);  // a row wholly inside this thread
        }
        h = same ? (h | hit[k]) : hit[k];
      }
      uint32_t lr = kNoRow, lh = 0;
      if (r7 == r0) fh = h;
      else { lr = r7; lh = h; }
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const uint32_t r = side ? lr : r0;
        bool head;
        const uint32_t rm = run_mask(r, &head);
        const uint32_t q = __reduce_or_sync(rm, side ? lh : fh);
        if (head && r != kNoRow && q) activate(r);
      }
      continue;
    }
    uint32_t uw[kEdgesPerThread], rw[kEdgesPerThread];
#pragma unroll
    for (int k = 0; k < kEdgesPerThread; ++k) {
      if (row[k] != kNoRow && (src[k] >= a.n_rows || row[k] >= a.n_rows)) {
        raise_error(a.ctr, kErrIndex);
        row[k] = kNoRow;
      }
      uw[k] = row[k] != kNoRow ? a.U[src[k] >> 5] : 0u;
      // The row's own changed bit, read at row starts only.
      const bool start = row[k] != kNoRow && row[k] != (k ? row[k - 1] : prev);
      rw[k] = start ? a.U[row[k] >> 5] : 0u;
    }
    uint32_t seg = kNoRow, hit = 0, first_row = kNoRow, first_hit = 0;
    bool first_open = true;
#pragma unroll
    for (int k = 0; k < kEdgesPerThread; ++k) {
      if (rw[k] && ((rw[k] >> (row[k] & 31u)) & 1u)) ++n_rows;
      if (row[k] == kNoRow) continue;
      if (row[k] != seg) {
        if (seg != kNoRow) {
          if (first_open) {
            first_row = seg;
            first_hit = hit;
            first_open = false;
          } else if (hit) {
            activate(seg);
          }
        }
        seg = row[k];
        hit = 0;
      }
      hit |= (uw[k] >> (src[k] & 31u)) & 1u;
    }
    uint32_t fr = seg, fh = hit, lr = kNoRow, lh = 0;
    if (!first_open) { fr = first_row; fh = first_hit; lr = seg; lh = hit; }
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const uint32_t r = side ? lr : fr;
      bool head;
      const uint32_t rm = run_mask(r, &head);
      const uint32_t q = __reduce_or_sync(rm, side ? lh : fh);
      if (head && r != kNoRow && q) activate(r);
    }
  }
  n_rows = __reduce_add_sync(kFull, (uint32_t)n_rows);
#pragma unroll
  for (int d = 16; d; d >>= 1) n_edges += __shfl_xor_sync(kFull, n_edges, d);
  if (lane == 0) {
    if (n_rows) atomicAdd(&a.ctr->updated, n_rows);
    if (n_edges) atomicAdd(&a.ctr->out_edges, n_edges);
  }
}

}  // namespace kites_internal
