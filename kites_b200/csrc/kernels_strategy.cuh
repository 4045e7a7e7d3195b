// kernels_strategy.cuh -- the per-iteration strategies the selector picks
// from.  Every strategy turns the set U of vertices changed by the previous
// iteration into the next changed set U', updating V in place; they differ
// in how they find the work:
//   PLAIN     expand U into the frontier A = out-neighbours(U), then the
//             edge-balanced pull over A (k_expand_chunked + k_pull_chunked);
//   PUSH      compact U into a queue (the reference's bitmapStreamExtraction,
//             kites/device/utility_device_functions.cuh:156-183, which the
//             reference never calls) and relax each queued vertex's weighted
//             out-edges with atomicMin;
//   PULL_ALL  pull over every vertex, reading V[u] + w only for in-neighbours
//             u in U (no expansion, no frontier bitmap);
//   TPV1/4/8/32  expand U into A, then pull with a fixed number of threads
//             per active vertex (no row splitting).
// All strategies reach the same fixed point (min is monotone and the
// changed set is exact), so switching between them per iteration changes
// the running time, never the result.
#pragma once
#include "kernels.cuh"

namespace kites_internal {

// ---- queue compaction + frontier statistics ----------------------------------

// Q <- ids of set bits of U (LSB-first, warp-aggregated append); also the
// count and out-degree sum of U, the selector's frontier features.
__global__ void k_compact_queue(const uint32_t *__restrict__ U, uint64_t nwords,
                                const uint32_t *__restrict__ out_deg, uint32_t *Q,
                                run_counters *ctr) {
  const uint32_t lane = lane_id();
  unsigned long long cnt = 0, odeg = 0;
  for (uint64_t wbase = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ull; wbase < nwords;
       wbase += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t wi = wbase + lane;
    const uint32_t word = wi < nwords ? U[wi] : 0u;
    const uint32_t c = __popc(word);
    const uint32_t incl = warp_inclusive_scan(c);
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    if (total == 0) continue;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(&ctr->queue_len[0], (unsigned long long)total);
    base = __shfl_sync(kFull, base, 0);
    uint32_t o = (uint32_t)(base + incl - c);
    uint32_t bits = word;
    while (bits) {
      const uint32_t b = __ffs(bits) - 1;
      bits &= bits - 1;
      const uint32_t v = (uint32_t)(wi * 32 + b);
      Q[o++] = v;
      odeg += out_deg[v];
    }
    cnt += c;
  }
  odeg = warp_sum_u64(odeg);
  if (lane == 0 && odeg) atomicAdd(&ctr->out_edges, odeg);
  (void)cnt;
}

// ---- push ------------------------------------------------------------------

template <typename OffT>
struct push_args {
  const OffT *outR;
  const uint32_t *outC;
  const uint32_t *outE;
  const uint32_t *Q;
  uint32_t *V;
  uint32_t *Unext;
  run_counters *ctr;
};

// One warp per queued vertex u: lanes stride over u's out-edges.
template <int OP, typename OffT>
__global__ void __launch_bounds__(kBlock) k_push_queue(push_args<OffT> a) {
  if (a.ctr->done) return;
  const uint32_t lane = lane_id();
  const unsigned long long qn = a.ctr->queue_len[0];
  unsigned long long n_edges = 0;
  uint32_t n_chg = 0;
  bool any = false;
  for (unsigned long long i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < qn;
       i += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
    const uint32_t u = a.Q[i];
    const uint32_t du = a.V[u];
    const OffT b = a.outR[u], e = a.outR[u + 1];
    if (lane == 0) n_edges += (unsigned long long)(e - b);
    for (OffT j = b + lane; j < e; j += 32) {
      const uint32_t v = __ldcs(a.outC + j);
      const uint32_t w = op_reads_weights<OP>() ? __ldcs(a.outE + j) : 0u;
      const uint32_t nd = nbr_comp<OP>(du, w);
      if (nd < a.V[v] && nd < atomicMin(a.V + v, nd)) {
        const uint32_t bit = 1u << (v & 31u);
        if (!(atomicOr(a.Unext + (v >> 5), bit) & bit)) ++n_chg;
        any = true;
      }
    }
  }
  if (__any_sync(kFull, any) && lane == 0) a.ctr->update_flag = 1u;
  n_chg = __reduce_add_sync(kFull, n_chg);
  if (lane == 0) {
    if (n_edges) atomicAdd(&a.ctr->edges, n_edges);
    if (n_chg) atomicAdd(&a.ctr->changed, (unsigned long long)n_chg);
  }
}

// ---- filtered dense pull (PULL_ALL) ------------------------------------------

// Every row (pull_args::rd null) or the frontier's rows (PULL_CHANGED), each
// folding only in-edges from sources with a U bit (pull_args::U the
// previous changed set, pull_args::chg the next one).
template <int OP, typename OffT>
__global__ void __launch_bounds__(kBlock) k_pull_all(pull_args<OffT> a) {
  if (a.ctr->done) return;
  pull_chunks<OP, OffT, true>(a);
}

// ---- threads-per-vertex pulls over the frontier A -----------------------------

template <typename OffT>
struct pull_tpv_args {
  const OffT *R;
  const uint32_t *C;
  const uint32_t *E;
  uint32_t *V;
  const uint32_t *A;       // frontier (vertex bits)
  uint32_t *Unext;
  uint64_t nwords;
  run_counters *ctr;
};

// A warp takes one frontier word; its active vertices are dealt to groups
// of TPV lanes, each group walking one vertex's whole in-row with stride TPV
// and reducing with __reduce_min_sync over the group.
template <int OP, typename OffT, int TPV>
__global__ void __launch_bounds__(kBlock) k_pull_tpv(pull_tpv_args<OffT> a) {
  if (a.ctr->done) return;
  constexpr int G = 32 / TPV;  // vertices in flight per warp
  const uint32_t lane = lane_id();
  const uint32_t grp = lane / TPV, gl = lane % TPV;
  const uint32_t gmask = (TPV == 32) ? kFull : (((1u << TPV) - 1u) << (grp * TPV));
  unsigned long long n_act = 0, n_edges = 0, n_chg = 0;
  for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < a.nwords;
       w += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
    uint32_t mask = a.A[w];
    uint32_t upd_bits = 0;
    while (mask) {
      // Deal the next G active vertices to the G groups.
      uint32_t mine = 32u;
      uint32_t m2 = mask;
#pragma unroll
      for (int gg = 0; gg < G; ++gg) {
        if (!m2) break;
        const uint32_t b = __ffs(m2) - 1;
        m2 &= m2 - 1;
        if ((uint32_t)gg == grp) mine = b;
      }
      mask = m2;
      uint32_t acc = kInf, old = kInf;
      uint64_t v = 0;
      if (mine < 32u) {
        v = w * 32 + mine;
        const OffT b = a.R[v], e = a.R[v + 1];
        if (gl == 0) { n_act += 1; n_edges += (unsigned long long)(e - b); }
        old = a.V[v];
        for (OffT j = b + gl; j < e; j += TPV) {
          const uint32_t src = __ldcs(a.C + j);
          const uint32_t wv = op_reads_weights<OP>() ? __ldcs(a.E + j) : 0u;
          acc = min(acc, nbr_comp<OP>(a.V[src], wv));
        }
      }
      if (TPV > 1) acc = __reduce_min_sync(gmask, acc);
      if (mine < 32u && gl == 0 && acc < old) {
        a.V[v] = acc;
        upd_bits |= 1u << mine;
      }
    }
    upd_bits = __reduce_or_sync(kFull, upd_bits);
    if (upd_bits && lane == 0) {
      n_chg += __popc(upd_bits & ~atomicOr(a.Unext + w, upd_bits));
      a.ctr->update_flag = 1u;
    }
  }
  n_act = warp_sum_u64(n_act);
  n_edges = warp_sum_u64(n_edges);
  if (lane == 0) {
    if (n_act) atomicAdd(&a.ctr->active, n_act);
    if (n_edges) atomicAdd(&a.ctr->edges, n_edges);
    if (n_chg) atomicAdd(&a.ctr->changed, n_chg);
  }
}

// Clears two word ranges (the frontier scratch and the consumed changed set).
__global__ void k_clear_two(uint32_t *a, uint32_t *b, uint64_t words) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words;
       i += (uint64_t)gridDim.x * blockDim.x) {
    a[i] = 0u;
    b[i] = 0u;
  }
}

}  // namespace kites_internal
