// kernels_batch.cuh -- batched multi-source pull: K sources at once over a
// V x K vertex-major distance array D (D[v*K + k]).
//
// One in-edge read serves all K sources: a warp walks the active vertices
// of an edge-balanced chunk one at a time; it loads 32 (C, E) pairs with
// one coalesced load, then for each edge a group of lanes gathers the
// source vertex's whole K-wide row (64 B .. 1 KB, contiguous) and folds it
// into its running minima.  Each lane moves 8 values (32 bytes) of a row
// with one 256-bit load (ld.global.v8.b32, new with sm_100), so a row takes
// K/8 lanes and a warp step covers 32/(K/8) edges; four steps' rows are
// loaded before any is folded (16 source rows in flight per warp for
// K = 64).  The lane groups' minima of a row meet over shuffles.  A vertex
// whose in-edges span several chunks merges its partial rows with
// atomicMin, like the single-source kernel.
//
// Changed sectors.  A lane's 8 values are one 32-byte sector of a row; the
// pulls and the push record, per vertex, which sectors of its row they
// lowered (M, one bit per sector, K/8 bits).  The masked pull gathers of an
// in-neighbour's row only the sectors that changed in the previous
// iteration (in-edges from a source with no changed sector cost no gather
// at all), and the push relaxes only those.  That is exact: after every
// iteration each edge (u, v) and column k either has u's sector of k marked
// or already satisfies D[v][k] <= nbrComp(D[u][k], w) -- a pull or push that
// reads D[u][k] establishes it, a later change of D[u][k] marks the sector
// again, and values only decrease.  It needs a monotone nbrComp, so the
// masked strategies take the saturating operators (SSSP, BFS).
#pragma once
#include "kernels.cuh"

namespace kites_internal {

template <int K>
struct batch_shape {
  static constexpr int VPL = 8;          // values per lane: one 32-byte access
  static constexpr int LPE = K / VPL;    // lanes per edge (a K-wide row)
  static constexpr int EPW = 32 / LPE;   // edges per warp step
  // Sector bits of a row (bit kl = lane kl's 8 values).
  static constexpr uint32_t kSectors = LPE == 32 ? kFull : ((1u << LPE) - 1u);
  static_assert(K == 16 || K == 32 || K == 64 || K == 128 || K == 256, "K");
};

template <int VPL>
__device__ __forceinline__ void load_row(const uint32_t *p, uint32_t (&x)[VPL]) {
  if constexpr (VPL == 1) {
    x[0] = *p;
  } else if constexpr (VPL == 2) {
    const uint2 t = *reinterpret_cast<const uint2 *>(p);
    x[0] = t.x; x[1] = t.y;
  } else {
#pragma unroll
    for (int q = 0; q < VPL / 4; ++q) {
      const uint4 t = reinterpret_cast<const uint4 *>(p)[q];
      x[4 * q] = t.x; x[4 * q + 1] = t.y; x[4 * q + 2] = t.z; x[4 * q + 3] = t.w;
    }
  }
}

template <int VPL>
__device__ __forceinline__ void store_row(uint32_t *p, const uint32_t (&x)[VPL]) {
  if constexpr (VPL == 1) {
    *p = x[0];
  } else if constexpr (VPL == 2) {
    *reinterpret_cast<uint2 *>(p) = make_uint2(x[0], x[1]);
  } else {
#pragma unroll
    for (int q = 0; q < VPL / 4; ++q)
      reinterpret_cast<uint4 *>(p)[q] =
          make_uint4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
  }
}

// One 32-byte access per lane (the address is 32-byte aligned: rows start at
// multiples of K >= 16 values and each lane's slice at a multiple of 8).
// Rows are not allocated in L1: an SM rarely gathers the same row twice
// (22 % L1 hits at scale 22), and skipping L1 made the scale-24 step 5.6 %
// faster (85.6 against 90.7 ms for K = 64); hub rows still meet in L2.
__device__ __forceinline__ void load_row8(const uint32_t *p, uint32_t (&x)[8]) {
  asm volatile("ld.global.L1::no_allocate.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(x[0]), "=r"(x[1]), "=r"(x[2]), "=r"(x[3]), "=r"(x[4]), "=r"(x[5]),
                 "=r"(x[6]), "=r"(x[7])
               : "l"(p));
}
// The same 32 bytes through L1: the push reads one source row for each of
// its out-edges, so the repeats hit.
__device__ __forceinline__ void load_row8_l1(const uint32_t *p, uint32_t (&x)[8]) {
  asm volatile("ld.global.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(x[0]), "=r"(x[1]), "=r"(x[2]), "=r"(x[3]), "=r"(x[4]), "=r"(x[5]),
                 "=r"(x[6]), "=r"(x[7])
               : "l"(p));
}
__device__ __forceinline__ void store_row8(uint32_t *p, const uint32_t (&x)[8]) {
  asm volatile("st.global.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
               :: "l"(p), "r"(x[0]), "r"(x[1]), "r"(x[2]), "r"(x[3]), "r"(x[4]), "r"(x[5]),
                  "r"(x[6]), "r"(x[7]) : "memory");
}

// Source rows each lane group keeps in flight.  Four, at 64 registers and
// four CTAs per SM, spill 152 bytes per thread and still beat two rows
// without spills by 8 % (R-MAT scale 24, K = 64); six and eight spill more
// and are slower.
template <int K>
constexpr int rows_in_flight() { return 4; }

// Rows with at most this many in-edges in a chunk go to the short-row path
// of the unmasked pull (one lane group per row); the warp-wide path keeps
// EPW x rows_in_flight = 16 gathers in flight per step (K = 64) only for
// rows at least that long.  R-MAT scale 24, K = 64, learned + batched:
// 247.1 GTEPS with 16, 243.4 with 8, 236.4 without the short-row path.
constexpr int64_t kShortRow = 16;

template <typename OffT>
struct pull_batch_args {
  chunk_geom<OffT> g;
  const uint32_t *E;
  uint32_t *D;            // n x K
  const uint32_t *rd;     // read frontier (vertex bits); null = every row
  uint32_t *chg;          // changed vertices
  run_counters *ctr;
  const uint32_t *Mprev;  // masked pull: changed sectors of the previous iteration
  uint32_t *Mnext;        // sectors this pull lowers, or null
};

// Four CTAs (32 warps) per SM keep more source rows in flight than fewer,
// fatter warps; K = 256 rows need the registers of two.  kMasked: gather
// only the changed sectors of each in-neighbour's row (a.Mprev); the live
// in-edges of a 32-edge tile are packed first so that lane groups take
// only edges that gather something.
template <int OP, typename OffT, int K, bool kMasked = false>
__global__ void __launch_bounds__(kBlock, K >= 256 ? 2 : 4)
    k_pull_batch(pull_batch_args<OffT> a) {
  if (a.ctr->done) return;
  using S = batch_shape<K>;
  constexpr int kRowsInFlight = rows_in_flight<K>();
  __shared__ uint8_t s_slot[kWarpsPerBlock][32];   // masked: lane of the j-th live edge
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  const uint32_t sub = lane / S::LPE, kl = lane % S::LPE;
  unsigned long long n_act = 0, n_edges = 0, n_chg = 0;
  const uint64_t stride = (uint64_t)gridDim.x * kWarpsPerBlock;
  for (uint64_t ch = (uint64_t)blockIdx.x * kWarpsPerBlock + wib; ch < a.g.nchunks;
       ch += stride) {
    const int64_t item_lo = (int64_t)(ch * a.g.chunk_items);
    const int64_t item_hi = min(item_lo + (int64_t)a.g.chunk_items, (int64_t)a.g.n_items);
    const uint64_t v_first = a.g.chunk_v0[ch];
    uint64_t v_last = a.g.chunk_v0[ch + 1];
    if (v_last >= a.g.n_rows) v_last = a.g.n_rows - 1;
    for (uint64_t vb = v_first & ~31ull; vb <= v_last; vb += 32) {
      uint32_t mask = a.rd ? a.rd[vb >> 5] : kFull;
      if (vb < v_first) mask &= kFull << (uint32_t)(v_first - vb);
      if (v_last - vb < 31) mask &= kFull >> (31u - (uint32_t)(v_last - vb));
      uint32_t upd_bits = 0;
      if constexpr (!kMasked && S::EPW >= 2) {
        // Short rows (at most kShortRow in-edges in this chunk) take one lane
        // group each: EPW rows at a time, kRowsInFlight gathers each, where
        // the warp-wide path below would keep only the row's few gathers in
        // flight and pay its row overhead serially.
        int64_t my_lo = 0, my_hi = 0;
        bool my_whole = false, my_short = false, my_owned = false;
        if ((mask >> lane) & 1u) {
          const uint64_t v = vb + lane;
          const int64_t r0 = (int64_t)a.g.R[v], r1 = (int64_t)a.g.R[v + 1];
          my_lo = max(r0, item_lo - (int64_t)v - 1);
          my_hi = min(r1, item_hi - (int64_t)v - 1);
          my_whole = my_lo == r0 && my_hi == r1;
          my_short = my_hi > my_lo && my_hi - my_lo <= kShortRow;
          my_owned = (int64_t)v + r0 >= item_lo && (int64_t)v + r0 < item_hi;
        }
        const uint32_t short_mask = __ballot_sync(kFull, my_short);
        const uint32_t s_act = __reduce_add_sync(kFull, (my_short && my_owned) ? 1u : 0u);
        const uint32_t s_edges = __reduce_add_sync(kFull, my_short ? (uint32_t)(my_hi - my_lo) : 0u);
        if (lane == 0) {
          n_act += s_act;
          n_edges += s_edges;
        }
        mask &= ~short_mask;
        uint32_t sm = short_mask;
        while (sm) {
          // Lane group `sub` takes the sub-th lowest row left in sm.
          uint32_t pick = sm;
#pragma unroll
          for (int q = 0; q + 1 < S::EPW; ++q)
            if ((uint32_t)q < sub) pick &= pick - 1;
#pragma unroll
          for (int q = 0; q < S::EPW; ++q) sm &= sm - 1;
          const bool has = pick != 0u;
          const uint32_t b = has ? (uint32_t)(__ffs(pick) - 1) : 0u;
          const int64_t lo = __shfl_sync(kFull, my_lo, b);
          const int64_t hi = __shfl_sync(kFull, my_hi, b);
          const bool whole = __shfl_sync(kFull, my_whole ? 1u : 0u, b) != 0u;
          bool lane_upd = false;
          if (has) {
            uint32_t acc[S::VPL];
#pragma unroll
            for (int q = 0; q < S::VPL; ++q) acc[q] = kInf;
            for (int64_t e0 = lo; e0 < hi; e0 += kRowsInFlight) {
              uint32_t row[kRowsInFlight][S::VPL], wq[kRowsInFlight];
#pragma unroll
              for (int r = 0; r < kRowsInFlight; ++r) {
                const int64_t e = e0 + r;
                wq[r] = 0u;
                if (e < hi) {
                  const uint32_t u = __ldcs(a.g.C + e);
                  if (op_reads_weights<OP>()) wq[r] = __ldcs(a.E + e);
                  load_row8(a.D + (uint64_t)u * K + kl * S::VPL, row[r]);
                } else {
#pragma unroll
                  for (int q = 0; q < S::VPL; ++q) row[r][q] = kInf;
                }
              }
#pragma unroll
              for (int r = 0; r < kRowsInFlight; ++r) {
                if (e0 + r >= hi) continue;
#pragma unroll
                for (int q = 0; q < S::VPL; ++q)
                  acc[q] = min(acc[q], nbr_comp<OP>(row[r][q], wq[r]));
              }
            }
            uint32_t *dv = a.D + (vb + b) * K + kl * S::VPL;
            uint32_t cur[S::VPL];
            load_row8(dv, cur);
            if (whole) {
              bool any = false;
#pragma unroll
              for (int q = 0; q < S::VPL; ++q) {
                if (acc[q] < cur[q]) { cur[q] = acc[q]; any = true; }
              }
              if (any) { store_row8(dv, cur); lane_upd = true; }
            } else {
#pragma unroll
              for (int q = 0; q < S::VPL; ++q)
                if (acc[q] < cur[q] && acc[q] < atomicMin(dv + q, acc[q])) lane_upd = true;
            }
          }
          // Each lane group's first lane publishes the sectors it lowered
          // and its row's changed bit.
          const uint32_t gbits = (__ballot_sync(kFull, lane_upd) >> (sub * S::LPE)) & S::kSectors;
          if (gbits && kl == 0 && a.Mnext) atomicOr(a.Mnext + vb + b, gbits);
          upd_bits |= __reduce_or_sync(kFull, (gbits && kl == 0) ? (1u << b) : 0u);
        }
      }
      while (mask) {
        const uint32_t b = __ffs(mask) - 1;
        mask &= mask - 1;
        const uint64_t v = vb + b;
        const int64_t r0 = (int64_t)a.g.R[v], r1 = (int64_t)a.g.R[v + 1];
        const int64_t lo = max(r0, item_lo - (int64_t)v - 1);
        const int64_t hi = min(r1, item_hi - (int64_t)v - 1);
        const int64_t vpos = (int64_t)v + r0;
        if (lane == 0) n_act += (vpos >= item_lo && vpos < item_hi) ? 1 : 0;
        if (hi <= lo) continue;
        if (lane == 0) n_edges += (uint64_t)(hi - lo);
        const bool whole = lo == r0 && hi == r1;
        uint32_t acc[S::VPL];
#pragma unroll
        for (int q = 0; q < S::VPL; ++q) acc[q] = kInf;
        bool row_live = !kMasked;
        for (int64_t tile = lo; tile < hi; tile += 32) {
          const int64_t t = tile + lane;
          uint32_t ntile = (uint32_t)min((int64_t)32, hi - tile);
          uint32_t cC = 0, cE = 0, cM = 0;
          if (t < hi) {
            cC = __ldcs(a.g.C + t);
            if (op_reads_weights<OP>()) cE = __ldcs(a.E + t);
          }
          if constexpr (kMasked) {
            cM = t < hi ? a.Mprev[cC] : 0u;
            const uint32_t live = __ballot_sync(kFull, cM != 0u);
            if (cM) s_slot[wib][__popc(live & ((1u << lane) - 1u))] = (uint8_t)lane;
            __syncwarp();
            ntile = __popc(live);
            row_live = row_live || live != 0u;
          }
          // kRowsInFlight source rows per lane group are loaded before any
          // is folded.
          for (uint32_t jj = 0; jj < ntile; jj += S::EPW * kRowsInFlight) {
            uint32_t row[kRowsInFlight][S::VPL], wq[kRowsInFlight];
#pragma unroll
            for (int r = 0; r < kRowsInFlight; ++r) {
              const uint32_t j = jj + r * S::EPW + sub;
              const uint32_t src = kMasked ? (j < ntile ? (uint32_t)s_slot[wib][j] : 0u)
                                           : (j & 31u);
              // Every lane takes part in every shuffle (full mask), whether
              // or not its slot gathers anything.
              const uint32_t u = __shfl_sync(kFull, cC, src);
              wq[r] = __shfl_sync(kFull, cE, src);
              const uint32_t mu = kMasked ? __shfl_sync(kFull, cM, src) : kFull;
              bool take = j < ntile && ((mu >> kl) & 1u);
              if (kMasked && take && u >= a.g.n_rows) {  // never index with an id out of range
                raise_error(a.ctr, kErrIndex);
                take = false;
              }
              if (take) {
                load_row8(a.D + (uint64_t)u * K + kl * S::VPL, row[r]);
              } else {
#pragma unroll
                for (int q = 0; q < S::VPL; ++q) row[r][q] = kInf;
              }
            }
#pragma unroll
            for (int r = 0; r < kRowsInFlight; ++r) {
              if (jj + r * S::EPW + sub >= ntile) continue;
#pragma unroll
              for (int q = 0; q < S::VPL; ++q) acc[q] = min(acc[q], nbr_comp<OP>(row[r][q], wq[r]));
            }
          }
          if constexpr (kMasked) __syncwarp();  // s_slot is rewritten by the next tile
        }
        if (!row_live) continue;  // masked: no in-neighbour changed
#pragma unroll
        for (int d = S::LPE; d < 32; d <<= 1) {
#pragma unroll
          for (int q = 0; q < S::VPL; ++q) acc[q] = min(acc[q], __shfl_xor_sync(kFull, acc[q], d));
        }
        bool lane_upd = false;
        if (sub == 0) {
          uint32_t *dv = a.D + v * K + kl * S::VPL;
          uint32_t cur[S::VPL];
          load_row8(dv, cur);
          if (whole) {
            bool any = false;
#pragma unroll
            for (int q = 0; q < S::VPL; ++q) {
              if (acc[q] < cur[q]) { cur[q] = acc[q]; any = true; }
            }
            if (any) { store_row8(dv, cur); lane_upd = true; }
          } else {
#pragma unroll
            for (int q = 0; q < S::VPL; ++q)
              if (acc[q] < cur[q] && acc[q] < atomicMin(dv + q, acc[q])) lane_upd = true;
          }
        }
        // Lanes 0 .. LPE-1 (lane group 0) own the row's sectors.
        const uint32_t sec = __ballot_sync(kFull, lane_upd) & S::kSectors;
        if (sec) {
          upd_bits |= 1u << b;
          if (a.Mnext && lane == 0) atomicOr(a.Mnext + v, sec);
        }
      }
      if (upd_bits && lane == 0) {
        n_chg += __popc(upd_bits & ~atomicOr(a.chg + (vb >> 5), upd_bits));
        a.ctr->update_flag = 1u;
      }
    }
  }
  if (lane == 0) {
    if (n_act) atomicAdd(&a.ctr->active, n_act);
    if (n_edges) atomicAdd(&a.ctr->edges, n_edges);
    if (n_chg) atomicAdd(&a.ctr->changed, n_chg);
  }
}

// ---- masked push ---------------------------------------------------------

template <typename OffT>
struct push_batch_args {
  chunk_geom<OffT> g;     // out-CSR: rows are sources, C their targets
  const uint32_t *outE;   // weights in out-CSR order
  uint32_t *D;            // n x K
  const uint32_t *U;      // rows changed by the previous iteration
  const uint32_t *Mprev;  // their changed sectors
  uint32_t *chg;          // next changed set
  uint32_t *Mnext;        // sectors lowered here
  run_counters *ctr;
};

// Sparse changed sets: the out-edges of the changed rows, walked over the
// out-CSR's edge-balanced chunks (as k_expand_chunked walks them); a lane
// group takes one out-edge (u, v) and, for each changed sector of u, lowers
// D[v]'s sector with atomicMin where nbrComp(D[u], w) beats it.
template <int OP, typename OffT, int K>
__global__ void __launch_bounds__(kBlock) k_push_batch(push_batch_args<OffT> a) {
  if (a.ctr->done) return;
  using S = batch_shape<K>;
  __shared__ uint32_t s_ex[kWarpsPerBlock][32];
  __shared__ OffT s_lo[kWarpsPerBlock][32];
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  const uint32_t sub = lane / S::LPE, kl = lane % S::LPE;
  uint32_t *ex = s_ex[wib];
  OffT *lo_s = s_lo[wib];
  unsigned long long n_rows = 0, n_edges = 0, n_chg = 0;
  bool any = false;
  const uint64_t stride = (uint64_t)gridDim.x * kWarpsPerBlock;
  for (uint64_t ch = (uint64_t)blockIdx.x * kWarpsPerBlock + wib; ch < a.g.nchunks;
       ch += stride) {
    const int64_t item_lo = (int64_t)(ch * a.g.chunk_items);
    const int64_t item_hi = min(item_lo + (int64_t)a.g.chunk_items, (int64_t)a.g.n_items);
    const uint64_t r_first = a.g.chunk_v0[ch];
    uint64_t r_last = a.g.chunk_v0[ch + 1];
    if (r_last >= a.g.n_rows) r_last = a.g.n_rows - 1;
    for (uint64_t rb = r_first & ~31ull; rb <= r_last; rb += 32) {
      const uint32_t word = a.U[rb >> 5];
      if (word == 0) continue;
      const uint64_t r = rb + lane;
      const bool active = r >= r_first && r <= r_last && ((word >> lane) & 1u);
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
      for (uint32_t base = 0; base < total; base += 32) {
        // Lane i loads virtual out-edge base + i: target, weight, source row
        // and the source's changed sectors.
        const uint32_t i = base + lane;
        uint32_t tv = 0, tw = 0, tr = 0, tm = 0;
        if (i < total) {
          const uint32_t j = owner_of(ex, i);
          const OffT e = lo_s[j] + (OffT)(i - ex[j]);
          tv = __ldcs(a.g.C + e);
          if (op_reads_weights<OP>()) tw = __ldcs(a.outE + e);
          tr = (uint32_t)(rb + j);
          tm = a.Mprev[tr];
        }
        const uint32_t nwin = min(32u, total - base);
        for (uint32_t s0 = 0; s0 < nwin; s0 += S::EPW) {
          const uint32_t sl = (s0 + sub) & 31u;
          const uint32_t v = __shfl_sync(kFull, tv, sl);
          const uint32_t w = __shfl_sync(kFull, tw, sl);
          const uint32_t u = __shfl_sync(kFull, tr, sl);
          const uint32_t mu = __shfl_sync(kFull, tm, sl);
          bool lowered = false;
          if (s0 + sub < nwin && ((mu >> kl) & 1u)) {
            uint32_t du[S::VPL], cur[S::VPL];
            load_row8_l1(a.D + (uint64_t)u * K + kl * S::VPL, du);
            uint32_t *dv = a.D + (uint64_t)v * K + kl * S::VPL;
            load_row8(dv, cur);
#pragma unroll
            for (int q = 0; q < S::VPL; ++q) {
              const uint32_t nd = nbr_comp<OP>(du[q], w);
              if (nd < cur[q] && nd < atomicMin(dv + q, nd)) lowered = true;
            }
          }
          // The group's first lane publishes the sectors its lanes lowered.
          const uint32_t gbits =
              (__ballot_sync(kFull, lowered) >> (sub * S::LPE)) & S::kSectors;
          if (gbits && kl == 0) {
            atomicOr(a.Mnext + v, gbits);
            const uint32_t bit = 1u << (v & 31u);
            if (!(atomicOr(a.chg + (v >> 5), bit) & bit)) ++n_chg;
            any = true;
          }
        }
      }
      __syncwarp();
    }
  }
  if (__any_sync(kFull, any) && lane == 0) a.ctr->update_flag = 1u;
  n_rows = warp_sum_u64(n_rows);
  n_edges = warp_sum_u64(n_edges);
  n_chg = warp_sum_u64(n_chg);
  if (lane == 0) {
    if (n_rows) atomicAdd(&a.ctr->active, n_rows);
    if (n_edges) atomicAdd(&a.ctr->edges, n_edges);
    if (n_chg) atomicAdd(&a.ctr->changed, n_chg);
  }
}

// Strategy loops start from the changed set: D = INF except D[s_k * K + k]
// = 0, bit s_k in U and sector k / 8 of s_k in M.
__global__ void k_seed_batch_changed(uint32_t *D, uint32_t K, const uint32_t *__restrict__ sources,
                                     uint32_t *U, uint32_t *M) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  const uint32_t s = sources[k];
  D[(uint64_t)s * K + k] = 0u;
  atomicOr(U + (s >> 5), 1u << (s & 31u));
  atomicOr(M + s, 1u << (k / 8u));
}

// D = INF everywhere, D[s_k * K + k] = 0, frontier bits for every
// out-neighbour of every source.
template <typename OffT>
__global__ void k_seed_batch(uint32_t *D, uint32_t K, const uint32_t *__restrict__ sources,
                             const OffT *__restrict__ outR, const uint32_t *__restrict__ outC,
                             uint32_t *frontier) {
  const uint32_t k = blockIdx.x;
  const uint32_t s = sources[k];
  if (threadIdx.x == 0) D[(uint64_t)s * K + k] = 0u;
  for (OffT i = outR[s] + threadIdx.x; i < outR[s + 1]; i += blockDim.x) {
    const uint32_t t = outC[i];
    atomicOr(frontier + (t >> 5), 1u << (t & 31u));
  }
}

}  // namespace kites_internal
