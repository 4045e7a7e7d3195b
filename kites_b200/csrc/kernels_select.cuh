// kernels_select.cuh -- the learned per-iteration strategy selector.
//
// Inference is fused into the frontier-count kernel: one pass over the
// changed set U counts its vertices and sums their out- and in-degrees; the
// last block to finish turns the counts into 12 features, runs the
// 12 -> 32 -> 32 -> 4 FP32 MLP and picks the strategy class, falling back to
// PLAIN unless the predicted gain clears the margin.  With a conditional
// handle it also sets the value of the graph's switch node.
//
// The MLP regresses, for each class, log(time(class) / time(PLAIN)) of the
// next iteration.  Training (k_mlp_grad + k_mlp_adam) is full-batch Adam on
// MSE over iterations recorded by running every class from the same state.
#pragma once
#include "kernels.cuh"

namespace kites_internal {

constexpr int kFeat = 12, kH = 32, kClasses = 4;
constexpr int kOffMean = 0, kOffStd = kFeat, kOffW1 = 2 * kFeat, kOffB1 = kOffW1 + kH * kFeat,
              kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH, kOffW3 = kOffB2 + kH,
              kOffB3 = kOffW3 + kClasses * kH, kParams = kOffB3 + kClasses;  // 1628

struct select_acc {
  unsigned long long cnt, osum, isum;
  unsigned int omax, blocks_done;
  unsigned long long msum;   // batched: changed sectors of the changed rows
  unsigned int imax, pad;    // largest in-degree of a changed row
};

// Guard of the threads-per-vertex class: it walks each row with one group
// of at most 32 lanes, so a row of this many in-edges or more (a hub of a
// power-law graph) holds its group far longer than an edge-balanced chunk;
// the class is not picked while the changed set holds such a row, whatever
// the model predicts.
constexpr unsigned int kTpvMaxRow = 8192;

template <typename OffT>
struct select_args {
  const uint32_t *U;
  uint64_t nwords;
  const uint32_t *out_deg;
  const OffT *R;
  uint64_t n, m;
  run_counters *ctr;
  select_acc *acc;
  const float *params;       // kParams floats, or null (always PLAIN)
  float margin_log;          // log(1 + margin)
  float *feat_out;           // optional: features of iteration i at [i * kFeat]
  uint32_t feat_cap;
  cudaGraphConditionalHandle handle;
  int has_handle;
  // Batched loop: the changed sectors of every vertex (null otherwise) and
  // the sectors per row; feature 9 becomes the changed fraction of the
  // changed rows' sectors.
  const uint32_t *M;
  uint32_t sectors;
};

// x (kFeat, raw) -> out (kClasses): standardise, two ReLU layers, linear.
__device__ __forceinline__ void mlp_forward_warp(const float *P, const float *x, float *h1,
                                                 float *h2, float *out) {
  const uint32_t j = lane_id();
  float a = P[kOffB1 + j];
#pragma unroll
  for (int i = 0; i < kFeat; ++i)
    a += P[kOffW1 + j * kFeat + i] * ((x[i] - P[kOffMean + i]) / P[kOffStd + i]);
  h1[j] = fmaxf(a, 0.f);
  __syncwarp();
  a = P[kOffB2 + j];
#pragma unroll
  for (int i = 0; i < kH; ++i) a += P[kOffW2 + j * kH + i] * h1[i];
  h2[j] = fmaxf(a, 0.f);
  __syncwarp();
  if (j < kClasses) {
    a = P[kOffB3 + j];
#pragma unroll
    for (int i = 0; i < kH; ++i) a += P[kOffW3 + j * kH + i] * h2[i];
    out[j] = a;
  }
  __syncwarp();
}

__device__ __forceinline__ float log2p1(double x) { return (float)log2(1.0 + x); }

template <typename OffT>
__global__ void __launch_bounds__(256) k_select(select_args<OffT> a) {
  if (a.ctr->done) {
    if (a.has_handle && blockIdx.x == 0 && threadIdx.x == 0)
      cudaGraphSetConditional(a.handle, 0);  // PLAIN branch, which exits at once
    return;
  }
  __shared__ unsigned long long s_c[8], s_o[8], s_i[8], s_s[8];
  __shared__ unsigned int s_m[8], s_x[8];
  __shared__ bool last;
  __shared__ float x[kFeat], h1[kH], h2[kH], out[kClasses];
  unsigned long long c = 0, os = 0, is = 0, ms = 0;
  unsigned int om = 0, im = 0;
  const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
  // A warp reads 32 changed-set words at once (one coalesced load, so an
  // empty stretch costs one load per 32 words); for each non-empty word a
  // lane takes one bit, so the degree loads of its vertices are coalesced,
  // and the loads of up to 8 non-empty words are in flight together.
  const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t base = (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32;
       base < a.nwords; base += nwarps * 32) {
    const uint64_t wl = base + lane;
    const uint32_t word = wl < a.nwords ? a.U[wl] : 0u;
    uint32_t nz = __ballot_sync(kFull, word != 0u);
    while (nz) {
      constexpr int kRound = 8;
      uint32_t od[kRound];
      OffT r0[kRound], r1[kRound];
#pragma unroll
      for (int q = 0; q < kRound; ++q) {
        const uint32_t i = nz ? (uint32_t)(__ffs(nz) - 1) : 32u;
        nz &= nz - 1;
        const uint32_t bits = __shfl_sync(kFull, word, i & 31u);
        const bool on = i < 32u && ((bits >> lane) & 1u);
        const uint64_t v = (base + (i & 31u)) * 32 + lane;
        od[q] = on ? a.out_deg[v] : 0u;
        r0[q] = on ? a.R[v] : (OffT)0;
        r1[q] = on ? a.R[v + 1] : (OffT)0;
        if (a.M) ms += on ? (unsigned long long)__popc(a.M[v]) : 0ull;
        c += on ? 1u : 0u;
      }
#pragma unroll
      for (int q = 0; q < kRound; ++q) {
        os += od[q];
        om = max(om, od[q]);
        const unsigned long long deg = (unsigned long long)(r1[q] - r0[q]);
        is += deg;
        im = max(im, (unsigned int)min(deg, 0xFFFFFFFFull));
      }
    }
  }
  c = __reduce_add_sync(kFull, (uint32_t)c);
  om = __reduce_max_sync(kFull, om);
  im = __reduce_max_sync(kFull, im);
#pragma unroll
  for (int d = 16; d; d >>= 1) {
    os += __shfl_xor_sync(kFull, os, d);
    is += __shfl_xor_sync(kFull, is, d);
    ms += __shfl_xor_sync(kFull, ms, d);
  }
  if (lane == 0) {
    s_c[wid] = c; s_o[wid] = os; s_i[wid] = is; s_m[wid] = om; s_s[wid] = ms; s_x[wid] = im;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tc = 0, to = 0, ti = 0, ts = 0;
    unsigned int tm = 0, tx = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      tc += s_c[i]; to += s_o[i]; ti += s_i[i]; ts += s_s[i]; tm = max(tm, s_m[i]);
      tx = max(tx, s_x[i]);
    }
    if (tc) {
      atomicAdd(&a.acc->cnt, tc);
      atomicAdd(&a.acc->osum, to);
      atomicAdd(&a.acc->isum, ti);
      atomicMax(&a.acc->omax, tm);
      atomicMax(&a.acc->imax, tx);
      if (ts) atomicAdd(&a.acc->msum, ts);
    }
    __threadfence();
    last = atomicAdd(&a.acc->blocks_done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last || wid != 0) return;
  __threadfence();
  // Last block, warp 0: features, MLP, choice.
  if (lane == 0) {
    const double cnt = (double)atomicAdd(&a.acc->cnt, 0ull);
    const double osum = (double)atomicAdd(&a.acc->osum, 0ull);
    const double isum = (double)atomicAdd(&a.acc->isum, 0ull);
    const double omax = (double)atomicMax(&a.acc->omax, 0u);
    const double n = (double)a.n, m = (double)(a.m ? a.m : 1);
    x[0] = log2p1(cnt);
    x[1] = log2p1(osum);
    x[2] = log2p1(isum);
    x[3] = (float)(cnt / n);
    x[4] = (float)(osum / m);
    x[5] = log2p1(omax);
    x[6] = (float)a.ctr->iterations / 32.f;
    x[7] = log2p1(n);
    x[8] = log2p1(m);
    if (a.M) {
      const double msum = (double)atomicAdd(&a.acc->msum, 0ull);
      x[9] = (float)(cnt > 0 ? msum / (cnt * (double)a.sectors) : 0.0);
    } else {
      x[9] = (float)(m / n / 32.0);
    }
    x[10] = log2p1((double)a.ctr->last_edges);
    x[11] = log2p1((double)a.ctr->last_active);
    s_x[0] = atomicMax(&a.acc->imax, 0u);
    a.acc->cnt = a.acc->osum = a.acc->isum = a.acc->msum = 0ull;
    a.acc->omax = 0u;
    a.acc->imax = 0u;
    a.acc->blocks_done = 0u;
    const unsigned long long it = a.ctr->iterations;
    if (a.feat_out && it < a.feat_cap)
      for (int i = 0; i < kFeat; ++i) a.feat_out[it * kFeat + i] = x[i];
  }
  __syncwarp();
  uint32_t cls = 0;
  if (a.params) {
    mlp_forward_warp(a.params, x, h1, h2, out);
    if (lane == 0) {
      // Class 3 of the single-source selector is the threads-per-vertex
      // pull; the batched loop's class 3 (a masked pull) needs no guard.
      const bool tpv_ok = a.M || s_x[0] < kTpvMaxRow;
      uint32_t best = 1;
      for (uint32_t k = 2; k < kClasses; ++k)
        if ((k != 3 || tpv_ok) && out[k] < out[best]) best = k;
      cls = (out[best] < out[0] - a.margin_log) ? best : 0u;
    }
  }
  if (lane == 0) {
    a.ctr->sel = cls;
    if (a.has_handle) cudaGraphSetConditional(a.handle, cls);
  }
}

// ---- training -----------------------------------------------------------------

// Feature mean / std over the dataset into P (one block).
__global__ void k_mlp_standardise(const float *__restrict__ X, uint32_t n, float *P) {
  const uint32_t f = threadIdx.x;
  if (f >= (uint32_t)kFeat) return;
  double s = 0, s2 = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const double v = X[(uint64_t)i * kFeat + f];
    s += v;
    s2 += v * v;
  }
  const double mean = s / n, var = s2 / n - mean * mean;
  P[kOffMean + f] = (float)mean;
  P[kOffStd + f] = (float)(var > 1e-12 ? sqrt(var) : 1.0);
}

// Deterministic small uniform init of the weights (biases 0).
__global__ void k_mlp_init(float *P, uint64_t seed) {
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < kParams; i += blockDim.x * gridDim.x) {
    if (i < kOffW1) continue;
    float fan = 0.f;
    if (i < kOffB1) fan = kFeat;
    else if (i >= kOffW2 && i < kOffB2) fan = kH;
    else if (i >= kOffW3 && i < kOffB3) fan = kH;
    if (fan == 0.f) { P[i] = 0.f; continue; }
    uint64_t z = seed + (uint64_t)i * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const float u = (float)((z >> 40) * (1.0 / 16777216.0)) * 2.f - 1.f;
    P[i] = u * sqrtf(6.f / fan) * 0.5f;
  }
}

// One thread per sample: forward, MSE loss against Y (log time ratios),
// backward; gradients summed in shared memory, then into G.
__global__ void __launch_bounds__(128)
    k_mlp_grad(const float *__restrict__ X, const float *__restrict__ Y, uint32_t n,
               const float *__restrict__ P, float *G, float *loss) {
  __shared__ float sg[kParams];
  __shared__ float sp[kParams];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
    sg[i] = 0.f;
    sp[i] = P[i];
  }
  __syncthreads();
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (s < n) {
    float xn[kFeat], z1[kH], h1[kH], z2[kH], h2[kH];
#pragma unroll
    for (int i = 0; i < kFeat; ++i)
      xn[i] = (X[(uint64_t)s * kFeat + i] - sp[kOffMean + i]) / sp[kOffStd + i];
    for (int j = 0; j < kH; ++j) {
      float a = sp[kOffB1 + j];
#pragma unroll
      for (int i = 0; i < kFeat; ++i) a += sp[kOffW1 + j * kFeat + i] * xn[i];
      z1[j] = a;
      h1[j] = fmaxf(a, 0.f);
    }
    for (int j = 0; j < kH; ++j) {
      float a = sp[kOffB2 + j];
      for (int i = 0; i < kH; ++i) a += sp[kOffW2 + j * kH + i] * h1[i];
      z2[j] = a;
      h2[j] = fmaxf(a, 0.f);
    }
    float d3[kClasses];
    for (int k = 0; k < kClasses; ++k) {
      float a = sp[kOffB3 + k];
      for (int i = 0; i < kH; ++i) a += sp[kOffW3 + k * kH + i] * h2[i];
      const float e = a - Y[(uint64_t)s * kClasses + k];
      l += e * e;
      d3[k] = 2.f * e / (float)n;
    }
    float d2[kH];
    for (int i = 0; i < kH; ++i) {
      float g = 0.f;
      for (int k = 0; k < kClasses; ++k) {
        g += d3[k] * sp[kOffW3 + k * kH + i];
        atomicAdd(&sg[kOffW3 + k * kH + i], d3[k] * h2[i]);
      }
      d2[i] = z2[i] > 0.f ? g : 0.f;
    }
    for (int k = 0; k < kClasses; ++k) atomicAdd(&sg[kOffB3 + k], d3[k]);
    float d1[kH];
    for (int i = 0; i < kH; ++i) d1[i] = 0.f;
    for (int j = 0; j < kH; ++j) {
      if (d2[j] == 0.f) continue;
      atomicAdd(&sg[kOffB2 + j], d2[j]);
      for (int i = 0; i < kH; ++i) {
        d1[i] += d2[j] * sp[kOffW2 + j * kH + i];
        atomicAdd(&sg[kOffW2 + j * kH + i], d2[j] * h1[i]);
      }
    }
    for (int j = 0; j < kH; ++j) {
      const float g = z1[j] > 0.f ? d1[j] : 0.f;
      if (g == 0.f) continue;
      atomicAdd(&sg[kOffB1 + j], g);
      for (int i = 0; i < kFeat; ++i) atomicAdd(&sg[kOffW1 + j * kFeat + i], g * xn[i]);
    }
  }
  for (int d = 16; d; d >>= 1) l += __shfl_xor_sync(kFull, l, d);
  if (lane_id() == 0 && l != 0.f) atomicAdd(loss, l / (float)n);
  __syncthreads();
  for (int i = threadIdx.x; i < kParams; i += blockDim.x)
    if (i >= kOffW1 && sg[i] != 0.f) atomicAdd(&G[i], sg[i]);
}

// Adam on the weights (mean/std entries untouched); zeroes G.
__global__ void k_mlp_adam(float *P, float *G, float *Mm, float *Vv, float lr, float b1,
                           float b2, float eps, int step) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams || i < kOffW1) return;
  const float g = G[i];
  const float m = b1 * Mm[i] + (1.f - b1) * g;
  const float v = b2 * Vv[i] + (1.f - b2) * g * g;
  Mm[i] = m;
  Vv[i] = v;
  const float mh = m / (1.f - powf(b1, (float)step));
  const float vh = v / (1.f - powf(b2, (float)step));
  P[i] -= lr * mh / (sqrtf(vh) + eps);
  G[i] = 0.f;
}

// Keeps the class picked for the coming iteration (read back for stats).
__global__ void k_record_sel(const run_counters *c, uint8_t *rec, uint32_t cap) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && !c->done && c->iterations < cap)
    rec[c->iterations] = (uint8_t)c->sel;
}

// Neutral selector: zero weights, unit std -- every prediction is 0, so the
// margin test always falls back to PLAIN.
__global__ void k_mlp_neutral(float *P) {
  for (int i = threadIdx.x; i < kParams; i += blockDim.x)
    P[i] = (i >= kOffStd && i < kOffStd + kFeat) ? 1.f : 0.f;
}

// Seeds at distance 0.  as_changed: each seed's bit in the changed set (the
// strategy loops); otherwise the frontier bits of every seed's out-neighbour
// groups (the plain loop, like the example's pre-processing).
template <typename OffT>
__global__ void k_seed_many(uint32_t *V, const uint32_t *__restrict__ seeds, uint64_t n_seeds,
                            const OffT *__restrict__ outR, const uint32_t *__restrict__ outC,
                            uint32_t shift, uint32_t *bits, int as_changed) {
  for (uint64_t i = blockIdx.x; i < n_seeds; i += gridDim.x) {
    const uint32_t s = seeds[i];
    if (threadIdx.x == 0) {
      V[s] = 0u;
      if (as_changed) atomicOr(bits + (s >> 5), 1u << (s & 31u));
    }
    if (!as_changed)
      for (OffT j = outR[s] + threadIdx.x; j < outR[s + 1]; j += blockDim.x) {
        const uint32_t gbit = outC[j] >> shift;
        atomicOr(bits + (gbit >> 5), 1u << (gbit & 31u));
      }
  }
}

// Sets V[source] = 0 and the source's bit in the changed set.
__global__ void k_seed_changed(uint32_t *V, uint32_t source, uint32_t *U) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    V[source] = 0u;
    U[source >> 5] |= 1u << (source & 31u);
  }
}

}  // namespace kites_internal
