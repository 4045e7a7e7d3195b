// kernels_batch_tma.cuh -- batched multi-source pull with TMA row gathers.
//
// The batched pull reads, for every in-edge (u -> v) of an active row, the
// K-wide source row D[u*K .. u*K + K) (128 B .. 1 KB).  With plain loads the
// bytes a warp keeps in flight are bounded by its registers; here each warp
// has its rows fetched by the Tensor Memory Accelerator instead:
// `cp.async.bulk.tensor.2d ... tile::gather4` copies four rows of D (given
// four row indices) into shared memory per instruction, completing on an
// mbarrier, so a warp keeps a whole group of G rows (8 KB) in flight while it
// folds the previous group out of shared memory.
//
// Work is the edge-balanced chunk table of the batched path (a warp per
// chunk).  A chunk's active rows (frontier bit set) form a stream of slots:
// for each row with in-edges in the chunk, one "own" slot -- the row's own
// D row, whose current values the fold compares against, so finalising a
// row needs no extra load -- then one slot per in-edge.  Slots are cut into
// groups of G (rows may span groups); the warp generates group g+1 (C and E
// loads, gathers issued by lane 0) before it waits for and folds group g.
// Lane l owns columns [l*VPL, l*VPL + VPL) of every row.  A row whose items
// all lie in the chunk has this warp as its only writer and is stored;
// a split row merges with atomicMin.
//
// Every mbarrier wait is bounded: after kTmaSpin unsuccessful rounds the
// warp records an error in the run counters, waits (bounded again) for its
// own copies still in flight and stops.
#pragma once
#include <cuda.h>

#include "kernels_batch.cuh"

namespace kites_internal {

constexpr int kTmaWarps = 4;                // warps per CTA
constexpr uint32_t kTmaSpin = 1u << 18;     // try_wait rounds (each <= ~1 us) before giving up

template <int K>
struct tma_batch_shape {
  static_assert(K == 32 || K == 64 || K == 128 || K == 256, "the TMA batched pull takes K >= 32");
  static constexpr int VPL = K / 32;                        // values per lane
  static constexpr int ROW = K * 4;                         // bytes per row of D
  static constexpr int G = 8192 / ROW < 32 ? 8192 / ROW : 32;  // slots per group
  static constexpr int BUF = G * ROW;                       // bytes per group buffer
  static_assert(G % 4 == 0, "groups are whole gather4 copies");
};

template <typename OffT>
struct tma_warp_meta {
  uint64_t bar[2];
  uint32_t ex[32];
  OffT lo[32];
};

template <int K, typename OffT>
constexpr size_t tma_batch_smem_bytes() {
  return (size_t)kTmaWarps * 2 * tma_batch_shape<K>::BUF +
         (size_t)kTmaWarps * sizeof(tma_warp_meta<OffT>);
}

template <typename OffT>
struct tma_batch_args {
  chunk_geom<OffT> g;
  const uint32_t *E;
  uint32_t *D;            // n x K
  const uint32_t *rd;     // read frontier (vertex bits)
  uint32_t *chg;          // changed vertices
  run_counters *ctr;
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// One bounded round of waiting for phase `parity` of the barrier (the
// thread may be suspended up to ~1 us inside try_wait).
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity), "r"(1000u)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (uint32_t i = 0; i < kTmaSpin; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Rows r0..r3 of the map (x = 0, the whole K-wide row each) into 4 * ROW
// consecutive bytes at dst; completes `bytes` on bar.
__device__ __forceinline__ void tma_gather4(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int32_t r0, int32_t r1, int32_t r2, int32_t r3) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(0), "r"(r0), "r"(r1),
      "r"(r2), "r"(r3)
      : "memory");
}

template <int VPL>
__device__ __forceinline__ void load_row_shared(const unsigned char *p, uint32_t (&x)[VPL]) {
  if constexpr (VPL == 1) {
    x[0] = *reinterpret_cast<const uint32_t *>(p);
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

template <int OP, typename OffT, int K>
__global__ void __launch_bounds__(kTmaWarps * 32)
    k_pull_batch_tma(const __grid_constant__ CUtensorMap dmap, tma_batch_args<OffT> a) {
  if (a.ctr->done) return;
  using S = tma_batch_shape<K>;
  constexpr int VPL = S::VPL;
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  constexpr bool kW = op_reads_weights<OP>();
  extern __shared__ __align__(1024) unsigned char smem[];
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  unsigned char *bufs = smem + (size_t)wib * 2 * S::BUF;
  tma_warp_meta<OffT> &mt = reinterpret_cast<tma_warp_meta<OffT> *>(
      smem + (size_t)kTmaWarps * 2 * S::BUF)[wib];
  if (lane == 0) {
    mbar_init(&mt.bar[0]);
    mbar_init(&mt.bar[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();

  uint32_t phase = 0u;      // bit b: parity to wait for next on buffer b
  uint32_t in_flight = 0u;  // bit b: buffer b has copies outstanding
  bool ok = true;
  int nb = 0;                       // buffer the next group goes to
  int pend = -1;                    // buffer of the group waiting to be folded
  uint32_t pend_n = 0;
  uint32_t p_row = kNone, p_w = 0;  // slot metadata of the pending group (lane i: slot i)
  bool p_own = false, p_skip = false;
  // The row being folded (carried across groups).
  uint32_t cur_row = kNone;
  bool cur_whole = false;
  uint32_t old[VPL], acc[VPL];
  uint32_t chg_word = kNone, chg_bits = 0;  // lane 0: changed bits not yet written
  unsigned long long n_act = 0, n_edges = 0, n_chg = 0;

  auto flush = [&]() {
    if (cur_row == kNone) return;
    bool imp = false;
    uint32_t *dv = a.D + (uint64_t)cur_row * K + lane * VPL;
    if (cur_whole) {
      uint32_t nv[VPL];
#pragma unroll
      for (int q = 0; q < VPL; ++q) {
        nv[q] = min(acc[q], old[q]);
        imp |= acc[q] < old[q];
      }
      if (imp) store_row<VPL>(dv, nv);
    } else {
#pragma unroll
      for (int q = 0; q < VPL; ++q)
        if (acc[q] < old[q] && acc[q] < atomicMin(dv + q, acc[q])) imp = true;
    }
    if (__any_sync(kFull, imp) && lane == 0) {
      const uint32_t word = cur_row >> 5;
      if (word != chg_word) {
        if (chg_word != kNone) n_chg += __popc(chg_bits & ~atomicOr(a.chg + chg_word, chg_bits));
        chg_word = word;
        chg_bits = 0;
      }
      chg_bits |= 1u << (cur_row & 31u);
      a.ctr->update_flag = 1u;
    }
    cur_row = kNone;
  };

  auto fold = [&]() {
    if (pend < 0) return;
    const int b = pend;
    pend = -1;
    if (!ok) return;
    // Every lane waits (the wait makes the copied bytes visible to it); the
    // warp goes on only if all of them saw the phase complete.
    const bool got = mbar_wait(&mt.bar[b], (phase >> b) & 1u);
    if (!__all_sync(kFull, got)) {
      ok = false;
      if (lane == 0) raise_error(a.ctr, kErrWait);
      return;
    }
    phase ^= 1u << b;
    in_flight &= ~(1u << b);
    const unsigned char *bp = bufs + (size_t)b * S::BUF + lane * VPL * 4;
    for (uint32_t s = 0; s < pend_n; ++s) {
      const uint32_t srow = __shfl_sync(kFull, p_row, s);
      const uint32_t sw = __shfl_sync(kFull, p_w, s);
      const bool sown = __shfl_sync(kFull, p_own ? 1u : 0u, s) != 0u;
      const bool sskip = __shfl_sync(kFull, p_skip ? 1u : 0u, s) != 0u;
      uint32_t v[VPL];
      load_row_shared<VPL>(bp + (size_t)s * S::ROW, v);
      if (sown) {
        flush();
        cur_row = srow;
        cur_whole = sw != 0u;
#pragma unroll
        for (int q = 0; q < VPL; ++q) {
          old[q] = v[q];
          acc[q] = kInf;
        }
      } else if (!sskip) {
#pragma unroll
        for (int q = 0; q < VPL; ++q) acc[q] = min(acc[q], nbr_comp<OP>(v[q], sw));
      }
    }
    __syncwarp();  // every lane is done reading buffer b before it is refilled
  };

  const uint64_t stride = (uint64_t)gridDim.x * kTmaWarps;
  for (uint64_t ch = (uint64_t)blockIdx.x * kTmaWarps + wib; ok && ch < a.g.nchunks;
       ch += stride) {
    const int64_t item_lo = (int64_t)(ch * a.g.chunk_items);
    const int64_t item_hi = min(item_lo + (int64_t)a.g.chunk_items, (int64_t)a.g.n_items);
    const uint64_t v_first = a.g.chunk_v0[ch];
    uint64_t v_last = a.g.chunk_v0[ch + 1];
    if (v_last >= a.g.n_rows) v_last = a.g.n_rows - 1;
    for (uint64_t vb = v_first & ~31ull; ok && vb <= v_last; vb += 32) {
      uint32_t mask = a.rd[vb >> 5];
      if (vb < v_first) mask &= kFull << (uint32_t)(v_first - vb);
      if (v_last - vb < 31) mask &= kFull >> (31u - (uint32_t)(v_last - vb));
      if (mask == 0) continue;
      // Lane j: row vb + j -- its slots (own + in-edges inside the chunk).
      const uint64_t v = vb + lane;
      uint32_t items = 0;
      OffT elo = 0;
      bool whole = false;
      if ((mask >> lane) & 1u) {
        const int64_t r0 = (int64_t)a.g.R[v], r1 = (int64_t)a.g.R[v + 1];
        const int64_t lo = max(r0, item_lo - (int64_t)v - 1);
        const int64_t hi = min(r1, item_hi - (int64_t)v - 1);
        const int64_t vpos = (int64_t)v + r0;
        n_act += (vpos >= item_lo && vpos < item_hi) ? 1u : 0u;
        if (hi > lo) {
          items = (uint32_t)(hi - lo) + 1u;
          n_edges += (uint64_t)(hi - lo);
          elo = (OffT)lo;
          whole = lo == r0 && hi == r1;
        }
      }
      const uint32_t incl = warp_inclusive_scan(items);
      const uint32_t total = __shfl_sync(kFull, incl, 31);
      if (total == 0) continue;
      const uint32_t whole_mask = __ballot_sync(kFull, whole);
      __syncwarp();
      mt.ex[lane] = incl - items;
      mt.lo[lane] = elo;
      __syncwarp();
      for (uint32_t base = 0; ok && base < total; base += S::G) {
        const uint32_t n = min((uint32_t)S::G, total - base);
        // Slot metadata: lane i < n holds slot base + i.
        uint32_t s_src = 0, s_row = kNone, s_w = 0;
        bool s_own = false, s_skip = false;
        if (lane < n) {
          const uint32_t q = base + lane;
          const uint32_t j = owner_of(mt.ex, q);
          const uint32_t kk = q - mt.ex[j];
          s_row = (uint32_t)(vb + j);
          if (kk == 0) {
            s_own = true;
            s_src = s_row;
            s_w = (whole_mask >> j) & 1u;
          } else {
            const OffT e = mt.lo[j] + (OffT)(kk - 1);
            s_src = __ldcs(a.g.C + e);
            s_w = kW ? __ldcs(a.E + e) : 0u;
            if (s_src >= a.g.n_rows) {  // out of range: never gather it
              raise_error(a.ctr, kErrIndex);
              s_skip = true;
              s_src = s_row;
            }
          }
        }
        // Issue the group's gathers into buffer nb (its last reader, the
        // fold two groups back, ended with __syncwarp).
        const uint32_t ng = (n + 3) / 4;
        if (lane == 0) {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_expect_tx(&mt.bar[nb], ng * 4 * S::ROW);
        }
        unsigned char *dst = bufs + (size_t)nb * S::BUF;
        for (uint32_t gi = 0; gi < ng; ++gi) {
          const uint32_t i0 = 4 * gi;
          const int32_t r0 = (int32_t)__shfl_sync(kFull, s_src, min(i0, n - 1));
          const int32_t r1 = (int32_t)__shfl_sync(kFull, s_src, min(i0 + 1, n - 1));
          const int32_t r2 = (int32_t)__shfl_sync(kFull, s_src, min(i0 + 2, n - 1));
          const int32_t r3 = (int32_t)__shfl_sync(kFull, s_src, min(i0 + 3, n - 1));
          if (lane == 0) tma_gather4(dst + (size_t)gi * 4 * S::ROW, &dmap, &mt.bar[nb], r0, r1, r2, r3);
        }
        in_flight |= 1u << nb;
        fold();
        pend = nb;
        pend_n = n;
        p_row = s_row;
        p_w = s_w;
        p_own = s_own;
        p_skip = s_skip;
        nb ^= 1;
      }
    }
  }
  fold();
  flush();
  if (!ok) {
    // Let this warp's copies still in flight land before the CTA exits.
    for (int b = 0; b < 2; ++b)
      if ((in_flight >> b) & 1u) mbar_wait(&mt.bar[b], (phase >> b) & 1u);
  }
  if (lane == 0) {
    if (chg_word != kNone && chg_bits)
      n_chg += __popc(chg_bits & ~atomicOr(a.chg + chg_word, chg_bits));
    if (n_chg) atomicAdd(&a.ctr->changed, n_chg);
  }
  n_act = __reduce_add_sync(kFull, (uint32_t)n_act);
#pragma unroll
  for (int d = 16; d; d >>= 1) n_edges += __shfl_xor_sync(kFull, n_edges, d);
  if (lane == 0) {
    if (n_act) atomicAdd(&a.ctr->active, n_act);
    if (n_edges) atomicAdd(&a.ctr->edges, n_edges);
  }
}

}  // namespace kites_internal
