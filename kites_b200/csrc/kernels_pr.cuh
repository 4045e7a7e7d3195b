// kernels_pr.cuh -- FP32 PageRank over the edge-balanced chunk table.
// One Jacobi step: y[v] = sum_{u->v} x[u] with x[u] = PR(u) / outdeg(u),
// then PR(v) = (1-d)/n + d y[v].  Whole rows store their sum; rows split
// over several chunks add their partial sums atomically.
#pragma once
#include "kernels.cuh"

namespace kites_internal {

// Sum of `p` over this lane's run of equal owners, valid at the run head.
__device__ __forceinline__ float run_sum_to_head(float p, uint32_t owner, bool *head) {
  const uint32_t rm = run_mask(owner, head);
  const uint32_t end = 31u - __clz(rm);
  const uint32_t lane = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const float q = __shfl_down_sync(kFull, p, d);
    if (lane + d <= end) p += q;
  }
  return p;
}

template <typename OffT>
__global__ void __launch_bounds__(kBlock)
    k_pr_pull(chunk_geom<OffT> g, const float *__restrict__ x, float *__restrict__ y) {
  __shared__ uint32_t s_ex[kWarpsPerBlock][32];
  __shared__ OffT s_lo[kWarpsPerBlock][32];
  __shared__ float s_acc[kWarpsPerBlock][32];
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  uint32_t *ex = s_ex[wib];
  OffT *lo_s = s_lo[wib];
  float *acc_s = s_acc[wib];
  const uint64_t stride = (uint64_t)gridDim.x * kWarpsPerBlock;
  for (uint64_t ch = (uint64_t)blockIdx.x * kWarpsPerBlock + wib; ch < g.nchunks;
       ch += stride) {
    const int64_t item_lo = (int64_t)(ch * g.chunk_items);
    const int64_t item_hi = min(item_lo + (int64_t)g.chunk_items, (int64_t)g.n_items);
    const uint64_t v_first = g.chunk_v0[ch];
    uint64_t v_last = g.chunk_v0[ch + 1];
    if (v_last >= g.n_rows) v_last = g.n_rows - 1;
    for (uint64_t vb = v_first & ~31ull; vb <= v_last; vb += 32) {
      const uint64_t v = vb + lane;
      const bool in_range = v >= v_first && v <= v_last;
      uint32_t cnt = 0;
      OffT elo = 0;
      bool whole = false;
      if (in_range) {
        const int64_t r0 = (int64_t)g.R[v], r1 = (int64_t)g.R[v + 1];
        const int64_t lo = max(r0, item_lo - (int64_t)v - 1);
        const int64_t hi = min(r1, item_hi - (int64_t)v - 1);
        cnt = hi > lo ? (uint32_t)(hi - lo) : 0u;
        elo = (OffT)lo;
        whole = (lo == r0) && (hi == r1);
      }
      const uint32_t incl = warp_inclusive_scan(cnt);
      const uint32_t total = __shfl_sync(kFull, incl, 31);
      if (total == 0) continue;
      ex[lane] = incl - cnt;
      lo_s[lane] = elo;
      acc_s[lane] = 0.f;
      __syncwarp();
      for (uint32_t base = 0; base < total; base += 32) {
        const uint32_t i = base + lane;
        uint32_t owner = 32u;
        float p = 0.f;
        if (i < total) {
          uint32_t j = 0;
#pragma unroll
          for (uint32_t step = 16; step; step >>= 1)
            if (ex[j + step] <= i) j += step;
          owner = j;
          const OffT e = lo_s[j] + (OffT)(i - ex[j]);
          p = x[__ldcs(g.C + e)];
        }
        bool head;
        p = run_sum_to_head(p, owner, &head);
        if (head && owner < 32u) acc_s[owner] += p;
        __syncwarp();
      }
      if (cnt) {
        if (whole) y[v] = acc_s[lane];
        else atomicAdd(y + v, acc_s[lane]);
      }
      __syncwarp();
    }
  }
}

__global__ void k_pr_init(const uint32_t *__restrict__ out_deg, uint64_t n, uint64_t n_real,
                          float *__restrict__ inv_out, float *__restrict__ x,
                          float *__restrict__ y, float *__restrict__ pr) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t d = out_deg[v];
    const float inv = d ? 1.0f / (float)d : 0.0f;
    const float r = v < n_real ? 1.0f / (float)n_real : 0.0f;
    inv_out[v] = inv;
    pr[v] = r;
    x[v] = r * inv;
    y[v] = 0.0f;
  }
}

__global__ void k_pr_update(uint64_t n_real, float base, float damping,
                            const float *__restrict__ inv_out, float *__restrict__ x,
                            float *__restrict__ y, float *__restrict__ pr) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n_real;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const float r = base + damping * y[v];
    pr[v] = r;
    x[v] = r * inv_out[v];
    y[v] = 0.0f;
  }
}

}  // namespace kites_internal
