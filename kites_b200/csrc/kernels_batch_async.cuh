// kernels_batch_async.cuh -- the batched V x K pull with its source-row
// gathers issued as asynchronous copies into shared memory (cp.async, two
// 16-byte copies per lane and row, L1 bypassed).  A copy in flight holds no
// register, so each lane group keeps kAsyncRows source rows in flight where
// the register version (k_pull_batch) keeps four at 64 registers and
// spills.  The work split, folds, updates and changed-sector marks are
// k_pull_batch's (unmasked, and masked: only the changed sectors of each
// in-neighbour's row, the live in-edges of a tile packed first);
// kites_graph_set_batch_gather(g, 2) selects it.
//
// Each lane copies and later reads back only its own 32 bytes of each row
// slot, so a lane waits for its own copies (cp.async.wait_all) and no
// barrier is needed between the copies and the folds.
#pragma once
#include "kernels_batch.cuh"

namespace kites_internal {

// Source rows in flight per lane group.  Six, at 48 KB of row slots and 64
// registers, let four CTAs reside per SM (24 rows in flight per warp, 768
// per SM); eight at three CTAs hold as many rows but fewer warps: R-MAT
// scale 24, K = 64, learned + batched 306.0 against 288.8 GTEPS.
constexpr int kAsyncRows = 6;

// Dynamic shared memory per CTA: per warp, per row slot, 32 bytes per lane.
constexpr size_t async_batch_smem_bytes() {
  return (size_t)kWarpsPerBlock * kAsyncRows * 32 * 32;
}

__device__ __forceinline__ void cp_async_row8(uint4 *smem, const uint32_t *gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile(
      "cp.async.cg.shared.global [%0], [%1], 16;\n\t"
      "cp.async.cg.shared.global [%2], [%3], 16;" ::"r"(s),
      "l"(gmem), "r"(s + 16u), "l"(gmem + 4)
      : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

__device__ __forceinline__ void smem_row8(const uint4 *smem, uint32_t (&x)[8]) {
  const uint4 p = smem[0], q = smem[1];
  x[0] = p.x; x[1] = p.y; x[2] = p.z; x[3] = p.w;
  x[4] = q.x; x[5] = q.y; x[6] = q.z; x[7] = q.w;
}

template <int OP, typename OffT, int K, bool kMasked = false>
__global__ void __launch_bounds__(kBlock, 4) k_pull_batch_async(pull_batch_args<OffT> a) {
  if (a.ctr->done) return;
  using S = batch_shape<K>;
  static_assert(S::VPL == 8, "one 32-byte sector per lane");
  extern __shared__ uint4 s_rows[];   // [warp][slot][lane][2]
  __shared__ uint8_t s_slot[kWarpsPerBlock][32];   // masked: lane of the j-th live edge
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  const uint32_t sub = lane / S::LPE, kl = lane % S::LPE;
  // This lane's slot r: my + r * 64 (32 lanes x 2 uint4 per slot).
  uint4 *my = s_rows + ((size_t)wib * kAsyncRows * 32 + lane) * 2;
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
        // Short rows (at most kShortRow in-edges in this chunk): one lane
        // group each, kAsyncRows gathers in flight per group.
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
        const uint32_t s_edges =
            __reduce_add_sync(kFull, my_short ? (uint32_t)(my_hi - my_lo) : 0u);
        if (lane == 0) {
          n_act += s_act;
          n_edges += s_edges;
        }
        mask &= ~short_mask;
        uint32_t sm = short_mask;
        while (sm) {
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
            for (int64_t e0 = lo; e0 < hi; e0 += kAsyncRows) {
              uint32_t wq[kAsyncRows];
#pragma unroll
              for (int r = 0; r < kAsyncRows; ++r) {
                const int64_t e = e0 + r;
                wq[r] = 0u;
                if (e < hi) {
                  const uint32_t u = __ldcs(a.g.C + e);
                  if (op_reads_weights<OP>()) wq[r] = __ldcs(a.E + e);
                  cp_async_row8(my + r * 64, a.D + (uint64_t)u * K + kl * S::VPL);
                }
              }
              cp_async_wait_all();
#pragma unroll
              for (int r = 0; r < kAsyncRows; ++r) {
                if (e0 + r >= hi) continue;
                uint32_t x[S::VPL];
                smem_row8(my + r * 64, x);
#pragma unroll
                for (int q = 0; q < S::VPL; ++q) acc[q] = min(acc[q], nbr_comp<OP>(x[q], wq[r]));
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
          for (uint32_t jj = 0; jj < ntile; jj += S::EPW * kAsyncRows) {
            uint32_t wq[kAsyncRows];
            bool tk[kAsyncRows];
#pragma unroll
            for (int r = 0; r < kAsyncRows; ++r) {
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
              tk[r] = take;
              if (take) cp_async_row8(my + r * 64, a.D + (uint64_t)u * K + kl * S::VPL);
            }
            cp_async_wait_all();
#pragma unroll
            for (int r = 0; r < kAsyncRows; ++r) {
              if (!tk[r]) continue;
              uint32_t x[S::VPL];
              smem_row8(my + r * 64, x);
#pragma unroll
              for (int q = 0; q < S::VPL; ++q) acc[q] = min(acc[q], nbr_comp<OP>(x[q], wq[r]));
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

// ---- masked push with asynchronous copies ------------------------------------

// Out-edges in flight per lane group in k_push_batch_async.
constexpr int kPushRows = 3;

// Dynamic shared memory per CTA: per warp, per out-edge slot, the source's
// and the target's 32 bytes for each lane.
constexpr size_t async_push_smem_bytes() {
  return (size_t)kWarpsPerBlock * kPushRows * 2 * 32 * 32;
}

// The source row sector through L1 (the push reads one source row once per
// out-edge, so repeats hit there).
__device__ __forceinline__ void cp_async_row8_l1(uint4 *smem, const uint32_t *gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile(
      "cp.async.ca.shared.global [%0], [%1], 16;\n\t"
      "cp.async.ca.shared.global [%2], [%3], 16;" ::"r"(s),
      "l"(gmem), "r"(s + 16u), "l"(gmem + 4)
      : "memory");
}

// k_push_batch with kPushRows out-edges per lane group in flight: the
// source's changed sectors and the target's current sectors of each edge are
// copied into shared memory together (cp.async), then the edges are relaxed
// one after another with atomicMin where the candidate beats the copy.  A
// source lowered by an earlier edge of the same round is read before that
// lowering; it is in the next changed set with those sectors marked, so its
// out-edges are pushed again then (the masked push's invariant).
template <int OP, typename OffT, int K>
__global__ void __launch_bounds__(kBlock, 4) k_push_batch_async(push_batch_args<OffT> a) {
  if (a.ctr->done) return;
  using S = batch_shape<K>;
  static_assert(S::VPL == 8, "one 32-byte sector per lane");
  extern __shared__ uint4 s_push[];   // [warp][slot][source|target][lane][2]
  __shared__ uint32_t s_ex[kWarpsPerBlock][32];
  __shared__ OffT s_lo[kWarpsPerBlock][32];
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  const uint32_t sub = lane / S::LPE, kl = lane % S::LPE;
  uint32_t *ex = s_ex[wib];
  OffT *lo_s = s_lo[wib];
  // This lane's source slot r: my + r * 128; its target slot: my + r * 128 + 64.
  uint4 *my = s_push + ((size_t)wib * kPushRows * 2 * 32 + lane) * 2;
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
        for (uint32_t s0 = 0; s0 < nwin; s0 += S::EPW * kPushRows) {
          uint32_t vv[kPushRows], ww[kPushRows];
          bool tk[kPushRows];
#pragma unroll
          for (int q = 0; q < kPushRows; ++q) {
            const uint32_t idx = s0 + q * S::EPW + sub;
            const uint32_t sl = idx & 31u;
            // Every lane takes part in every shuffle (full mask).
            vv[q] = __shfl_sync(kFull, tv, sl);
            ww[q] = __shfl_sync(kFull, tw, sl);
            const uint32_t u = __shfl_sync(kFull, tr, sl);
            const uint32_t mu = __shfl_sync(kFull, tm, sl);
            tk[q] = idx < nwin && ((mu >> kl) & 1u);
            if (tk[q]) {
              cp_async_row8_l1(my + q * 128, a.D + (uint64_t)u * K + kl * S::VPL);
              cp_async_row8(my + q * 128 + 64, a.D + (uint64_t)vv[q] * K + kl * S::VPL);
            }
          }
          cp_async_wait_all();
#pragma unroll
          for (int q = 0; q < kPushRows; ++q) {
            bool lowered = false;
            if (tk[q]) {
              uint32_t du[S::VPL], cur[S::VPL];
              smem_row8(my + q * 128, du);
              smem_row8(my + q * 128 + 64, cur);
              uint32_t *dv = a.D + (uint64_t)vv[q] * K + kl * S::VPL;
#pragma unroll
              for (int x = 0; x < S::VPL; ++x) {
                const uint32_t nd = nbr_comp<OP>(du[x], ww[q]);
                if (nd < cur[x] && nd < atomicMin(dv + x, nd)) lowered = true;
              }
            }
            // The group's first lane publishes the sectors its lanes lowered.
            const uint32_t gbits =
                (__ballot_sync(kFull, lowered) >> (sub * S::LPE)) & S::kSectors;
            if (gbits && kl == 0) {
              atomicOr(a.Mnext + vv[q], gbits);
              const uint32_t bit = 1u << (vv[q] & 31u);
              if (!(atomicOr(a.chg + (vv[q] >> 5), bit) & bit)) ++n_chg;
              any = true;
            }
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

}  // namespace kites_internal
