// engine.cu -- C ABI of the B200 vertex-centric engine: engine/graph
// lifetimes, device layout build, and the iteration loops of the built-in
// vertex programs (host-driven as in kites/device/compute.cuh:57-128, or a
// CUDA graph with a conditional while node and device-side convergence).
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "engine.cuh"
#include "kernels.cuh"
#include "kernels_batch.cuh"
#include "kernels_batch_async.cuh"
#include "kernels_batch_tma.cuh"
#include "kernels_mip.cuh"
#include "kernels_pr.cuh"
#include "kernels_select.cuh"
#include "kernels_strategy.cuh"
#include "kernels_sweep.cuh"

using namespace kites_internal;

namespace kites_internal {

char *error_buffer() {
  static thread_local char buf[512];
  return buf;
}

namespace {

// Default selector weights: written by `python -m kites_b200.train_selector
// --inc`, trained on generated graphs; without the file a fresh engine has
// neutral weights (always PLAIN).
#if __has_include("selector_default.inc")
#define KITES_HAVE_DEFAULT_SELECTOR 1
static const float kDefaultSelector[] = {
#include "selector_default.inc"
};
static_assert(sizeof(kDefaultSelector) == kParams * sizeof(float),
              "selector_default.inc must hold the 1628 selector parameters");
#endif
// The batched loop's selector (classes PLAIN, PUSH, PULL_ALL, PULL_CHANGED),
// written by `python -m kites_b200.train_selector --batch --inc ...`.
#if __has_include("selector_batch_default.inc")
#define KITES_HAVE_DEFAULT_BATCH_SELECTOR 1
static const float kDefaultBatchSelector[] = {
#include "selector_batch_default.inc"
};
static_assert(sizeof(kDefaultBatchSelector) == kParams * sizeof(float),
              "selector_batch_default.inc must hold the 1628 selector parameters");
#endif

int dev_alloc(kites_engine *eng, void **p, size_t bytes) {
  *p = nullptr;
  // At least 16 bytes of slack past the end: the staged sweep copies whole
  // 16-byte pieces, so a slice ending inside the last piece reads up to 12
  // bytes beyond the array.
  bytes = (bytes + 16 + 255) & ~size_t(255);
  cudaError_t e = cudaMallocFromPoolAsync(p, bytes, eng->pool, eng->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(KITES_ERR_OOM, "device pool allocation of %zu bytes failed: %s",
                bytes, cudaGetErrorString(e));
  }
  return KITES_OK;
}

// Status of a run that a kernel stopped (run_counters::error bits).  A wait
// that gave up is a timeout; an out-of-range index read during the run means
// the device arrays no longer hold what the upload validated.
int run_error(uint32_t err) {
  if (err & kErrWait)
    return fail(KITES_ERR_TIMEOUT,
                "a bounded wait on a TMA row copy gave up (error bits 0x%x)", err);
  return fail(KITES_ERR_CUDA,
              "a kernel read an out-of-range vertex or edge index and skipped it "
              "(error bits 0x%x)", err);
}

int graph_alloc(kites_graph *g, void **p, size_t bytes) {
  KITES_TRY(dev_alloc(g->eng, p, bytes));
  g->owned.push_back(*p);
  return KITES_OK;
}

inline unsigned grid_for(uint64_t n, unsigned block = 256, unsigned cap = 65535u * 8) {
  uint64_t b = (n + block - 1) / block;
  if (b == 0) b = 1;
  return (unsigned)(b > cap ? cap : b);
}

int set_device(kites_engine *eng) {
  KITES_CUDA_TRY(cudaSetDevice(eng->device));
  return KITES_OK;
}

template <typename OffT>
int build_chunk_table(kites_graph *g, const OffT *R, uint64_t n_rows,
                      uint64_t n_edges, uint32_t **table, uint64_t *nchunks) {
  const uint64_t items = n_rows + n_edges;
  uint64_t nc = (items + g->chunk_items - 1) / g->chunk_items;
  if (nc == 0) nc = 1;
  void *p;
  KITES_TRY(graph_alloc(g, &p, (nc + 1) * sizeof(uint32_t)));
  *table = (uint32_t *)p;
  *nchunks = nc;
  if (n_rows == 0) {
    KITES_CUDA_TRY(cudaMemsetAsync(p, 0, (nc + 1) * sizeof(uint32_t), g->eng->stream));
    return KITES_OK;
  }
  k_chunk_table<OffT><<<grid_for(nc + 1), 256, 0, g->eng->stream>>>(
      R, n_rows, nc, g->chunk_items, *table);
  KITES_CUDA_TRY(cudaGetLastError());
  return KITES_OK;
}

// Device row offsets of type OffT with n_rows+1 entries from a host/device
// source of n_src+1 entries (uint64 or uint32); rows past n_src repeat the
// last offset (empty padding rows).
template <typename OffT>
int upload_offsets(kites_graph *g, const uint64_t *src64, const uint32_t *src32,
                   uint64_t n_src, uint64_t n_rows, int on_device, OffT **out) {
  kites_engine *eng = g->eng;
  void *p;
  KITES_TRY(graph_alloc(g, &p, (n_rows + 1) * sizeof(OffT)));
  OffT *R = (OffT *)p;
  const bool same = (src64 && sizeof(OffT) == 8) || (src32 && sizeof(OffT) == 4);
  if (same) {
    const void *src = src64 ? (const void *)src64 : (const void *)src32;
    KITES_CUDA_TRY(cudaMemcpyAsync(R, src, (n_src + 1) * sizeof(OffT),
                                   cudaMemcpyDefault, eng->stream));
  } else {
    void *tmp;
    const size_t esz = src64 ? 8 : 4;
    KITES_TRY(dev_alloc(eng, &tmp, (n_src + 1) * esz));
    KITES_CUDA_TRY(cudaMemcpyAsync(tmp, src64 ? (const void *)src64 : (const void *)src32,
                                   (n_src + 1) * esz, cudaMemcpyDefault, eng->stream));
    if (src64)
      k_narrow_offsets<OffT><<<grid_for(n_src + 1), 256, 0, eng->stream>>>(
          (const uint64_t *)tmp, n_src + 1, R);
    else
      k_widen_offsets<OffT><<<grid_for(n_src + 1), 256, 0, eng->stream>>>(
          (const uint32_t *)tmp, n_src + 1, R);
    KITES_CUDA_TRY(cudaGetLastError());
    KITES_CUDA_TRY(cudaFreeAsync(tmp, eng->stream));
  }
  (void)on_device;
  if (n_rows > n_src) {
    // Fill R[n_src+1 .. n_rows] with R[n_src] (read back on device).
    pad_offsets<OffT><<<grid_for(n_rows - n_src), 256, 0, eng->stream>>>(R, n_src, n_rows);
    KITES_CUDA_TRY(cudaGetLastError());
  }
  *out = R;
  return KITES_OK;
}


// Checks offsets and ids on the device before anything traverses them.
template <typename OffT>
int validate_csc(kites_graph *g, const OffT *R, uint64_t n_rows, uint64_t n_edges,
                 const uint32_t *ids, uint64_t limit, const char *what) {
  kites_engine *eng = g->eng;
  cudaStream_t s = eng->stream;
  void *p;
  KITES_TRY(dev_alloc(eng, &p, 4));
  uint32_t *bad = (uint32_t *)p;
  KITES_CUDA_TRY(cudaMemsetAsync(bad, 0, 4, s));
  if (n_rows) k_validate_rows<OffT><<<grid_for(n_rows), 256, 0, s>>>(R, n_rows, n_edges, bad);
  if (n_edges) k_validate_ids<<<grid_for(n_edges), 256, 0, s>>>(ids, n_edges, limit, bad);
  KITES_CUDA_TRY(cudaGetLastError());
  uint32_t *h = (uint32_t *)eng->pinned;
  KITES_CUDA_TRY(cudaMemcpyAsync(h, bad, 4, cudaMemcpyDeviceToHost, s));
  KITES_CUDA_TRY(cudaFreeAsync(bad, s));
  KITES_CUDA_TRY(cudaStreamSynchronize(s));
  if (*h & 1u)
    return fail(KITES_ERR_INVALID, "%s offsets are not 0..n_edges non-decreasing", what);
  if (*h & 2u)
    return fail(KITES_ERR_INVALID, "%s has an index >= %llu", what, (unsigned long long)limit);
  return KITES_OK;
}

// Weighted vertex-level out-CSR from the CSC: stable radix sort of the edge
// indices by source keeps destinations ascending within each out-row.
template <typename OffT>
int build_out_csr(kites_graph *g) {
  kites_engine *eng = g->eng;
  cudaStream_t s = eng->stream;
  const uint64_t n = g->n, m = g->m;
  const OffT *R = (const OffT *)g->R;
  void *p;
  KITES_TRY(graph_alloc(g, &p, (n + 1) * sizeof(OffT)));
  g->outR = p;
  KITES_TRY(graph_alloc(g, &p, m * sizeof(uint32_t)));
  g->outC = (uint32_t *)p;
  KITES_TRY(graph_alloc(g, &p, m * sizeof(uint32_t)));
  g->outE = (uint32_t *)p;
  KITES_TRY(graph_alloc(g, &p, (n + 1) * sizeof(uint32_t)));
  g->out_deg = (uint32_t *)p;
  KITES_CUDA_TRY(cudaMemsetAsync(g->out_deg, 0, (n + 1) * sizeof(uint32_t), s));
  // The transposition sorts 32-bit edge ids (item counts are 64-bit).
  if (m > 0xFFFFFFFFull)
    return fail(KITES_ERR_UNSUPPORTED, "out-CSR build supports < 2^32 edges");
  if (m) {
    k_count_u32<<<grid_for(m), 256, 0, s>>>(g->C, m, g->out_deg);
    KITES_CUDA_TRY(cudaGetLastError());
  }
  // outR = exclusive scan of out-degrees (as OffT).
  OffT *deg_wide;
  KITES_TRY(dev_alloc(eng, &p, (n + 1) * sizeof(OffT)));
  deg_wide = (OffT *)p;
  k_widen_offsets<OffT><<<grid_for(n + 1), 256, 0, s>>>(g->out_deg, n + 1, deg_wide);
  size_t temp_bytes = 0;
  KITES_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, deg_wide,
                                               (OffT *)g->outR, (uint64_t)(n + 1), s));
  void *temp;
  KITES_TRY(dev_alloc(eng, &temp, temp_bytes));
  KITES_CUDA_TRY(cub::DeviceScan::ExclusiveSum(temp, temp_bytes, deg_wide,
                                               (OffT *)g->outR, (uint64_t)(n + 1), s));
  KITES_CUDA_TRY(cudaFreeAsync(temp, s));
  KITES_CUDA_TRY(cudaFreeAsync(deg_wide, s));
  if (m == 0) return KITES_OK;

  uint32_t *row, *keys_out, *idx_in, *idx_out;
  KITES_TRY(dev_alloc(eng, &p, m * 4)); row = (uint32_t *)p;
  KITES_TRY(dev_alloc(eng, &p, m * 4)); keys_out = (uint32_t *)p;
  KITES_TRY(dev_alloc(eng, &p, m * 4)); idx_in = (uint32_t *)p;
  KITES_TRY(dev_alloc(eng, &p, m * 4)); idx_out = (uint32_t *)p;
  k_row_of_edge<OffT><<<grid_for(m), 256, 0, s>>>(R, n + 1, m, row);
  k_iota_u32<<<grid_for(m), 256, 0, s>>>(idx_in, m);
  KITES_CUDA_TRY(cudaGetLastError());
  int end_bit = 1;
  while (end_bit < 32 && (1ull << end_bit) < n) ++end_bit;
  temp_bytes = 0;
  KITES_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, g->C, keys_out,
                                                 idx_in, idx_out, (uint64_t)m, 0, end_bit, s));
  KITES_TRY(dev_alloc(eng, &temp, temp_bytes));
  KITES_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, g->C, keys_out,
                                                 idx_in, idx_out, (uint64_t)m, 0, end_bit, s));
  k_gather_out<OffT><<<grid_for(m), 256, 0, s>>>(
      idx_out, row, g->esize == 4 ? (const uint32_t *)g->E : nullptr, m, g->outC, g->outE);
  KITES_CUDA_TRY(cudaGetLastError());
  KITES_CUDA_TRY(cudaFreeAsync(temp, s));
  KITES_CUDA_TRY(cudaFreeAsync(row, s));
  KITES_CUDA_TRY(cudaFreeAsync(keys_out, s));
  KITES_CUDA_TRY(cudaFreeAsync(idx_in, s));
  KITES_CUDA_TRY(cudaFreeAsync(idx_out, s));
  return KITES_OK;
}

template <typename OffT>
int upload_typed(kites_graph *g, const kites_csc_view *v) {
  kites_engine *eng = g->eng;
  cudaStream_t s = eng->stream;
  OffT *R;
  KITES_TRY(upload_offsets<OffT>(g, v->row_offsets, v->row_offsets32, v->n_vertices,
                                 g->n, v->on_device, &R));
  g->R = R;
  void *p;
  KITES_TRY(graph_alloc(g, &p, g->m * sizeof(uint32_t)));
  g->C = (uint32_t *)p;
  if (g->m)
    KITES_CUDA_TRY(cudaMemcpyAsync(g->C, v->col_indices, g->m * 4, cudaMemcpyDefault, s));
  KITES_TRY(validate_csc<OffT>(g, R, g->n, g->m, g->C, g->n_given, "CSC"));
  if (g->esize) {
    KITES_TRY(graph_alloc(g, &p, g->m * g->esize));
    g->E = p;
    if (g->m)
      KITES_CUDA_TRY(cudaMemcpyAsync(g->E, v->edge_values, g->m * g->esize,
                                     cudaMemcpyDefault, s));
  }
  KITES_TRY(graph_alloc(g, &p, g->n * g->vsize));
  g->V = p;
  KITES_CUDA_TRY(cudaMemsetAsync(g->V, 0, g->n * g->vsize, s));
  if (v->vertex_values)
    KITES_CUDA_TRY(cudaMemcpyAsync(g->V, v->vertex_values, v->n_vertices * g->vsize,
                                   cudaMemcpyDefault, s));

  // Out-CSR structure for every graph; its weights only mean something for
  // 4-byte edge values (other sizes get 1).
  KITES_TRY(build_out_csr<OffT>(g));

  // Activation adjacency.
  if (!g->directed) {
    g->dirR = g->R;
    g->dirC = g->C;
    g->n_dir_rows = g->n;
    g->n_dir_edges = g->m;
  } else if (g->vpg == 1) {
    if (!g->outR) return fail(KITES_ERR_UNSUPPORTED, "directed vpg=1 needs 4-byte edges");
    g->dirR = g->outR;
    g->dirC = g->outC;
    g->n_dir_rows = g->n;
    g->n_dir_edges = g->m;
  } else {
    if (!v->out_col_indices || (!v->out_row_offsets && !v->out_row_offsets32))
      return fail(KITES_ERR_INVALID, "vertex_per_group > 1 needs the group out-adjacency");
    OffT *dR;
    KITES_TRY(upload_offsets<OffT>(g, v->out_row_offsets, v->out_row_offsets32,
                                   v->n_out_rows, v->n_out_rows, v->on_device, &dR));
    g->dirR = dR;
    g->n_dir_rows = v->n_out_rows;
    g->n_dir_edges = v->n_out_edges;
    KITES_TRY(graph_alloc(g, &p, g->n_dir_edges * 4));
    g->dirC = (uint32_t *)p;
    if (g->n_dir_edges)
      KITES_CUDA_TRY(cudaMemcpyAsync(g->dirC, v->out_col_indices, g->n_dir_edges * 4,
                                     cudaMemcpyDefault, s));
    const uint64_t ngroups = (g->n + g->vpg - 1) / g->vpg;
    if (g->n_dir_rows > ngroups)
      return fail(KITES_ERR_INVALID, "group out-adjacency has %llu rows, graph has %llu groups",
                  (unsigned long long)g->n_dir_rows, (unsigned long long)ngroups);
    KITES_TRY(validate_csc<OffT>(g, dR, g->n_dir_rows, g->n_dir_edges, g->dirC, ngroups,
                                 "group out-adjacency"));
  }
  KITES_TRY(build_chunk_table<OffT>(g, (const OffT *)g->R, g->n, g->m, &g->chunk_in,
                                    &g->nchunks_in));
  if (g->dirR == g->R) {
    g->chunk_dir = g->chunk_in;
    g->nchunks_dir = g->nchunks_in;
  } else {
    KITES_TRY(build_chunk_table<OffT>(g, (const OffT *)g->dirR, g->n_dir_rows,
                                      g->n_dir_edges, &g->chunk_dir, &g->nchunks_dir));
  }

  int per_sm = 0;
  KITES_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, k_pull_chunked<OP_SSSP, OffT>, kBlock, 0));
  if (per_sm < 1) per_sm = 1;
  const uint64_t cap = (uint64_t)per_sm * eng->sm_count;
  uint64_t want = (g->nchunks_in + kWarpsPerBlock - 1) / kWarpsPerBlock;
  g->pull_grid = (int)(want < cap ? (want ? want : 1) : cap);
  want = (g->nchunks_dir + kWarpsPerBlock - 1) / kWarpsPerBlock;
  g->expand_grid = (int)(want < cap ? (want ? want : 1) : cap);

  // Edge-parallel dense sweeps: the row of every edge, persistent grid.
  if (g->vpg == 1) {
    if (g->m) {
      void *p;
      KITES_TRY(graph_alloc(g, &p, g->m * 4));
      g->rowid = (uint32_t *)p;
      k_row_of_edge<OffT><<<grid_for(g->m), 256, 0, eng->stream>>>((const OffT *)g->R, g->n + 1,
                                                                  g->m, g->rowid);
      KITES_CUDA_TRY(cudaGetLastError());
    }
    int per_sm_sweep = 0;
    KITES_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm_sweep, k_sweep<OP_SSSP, OffT, kRowFilter>, kSweepThreads, 0));
    const uint64_t scap = (uint64_t)std::max(per_sm_sweep, 1) * eng->sm_count;
    const uint64_t windows = (g->m + kWindowEdges - 1) / kWindowEdges;
    const uint64_t want_blocks = (windows + kSweepThreads / 32 - 1) / (kSweepThreads / 32);
    g->sweep_grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(want_blocks, scap));
    g->dense_edges = g->m / 16;
    g->dense_rows = g->n / 32;
  }
  return KITES_OK;
}

// ---- iteration loops ----------------------------------------------------

template <int OP, typename OffT, int MODE>
void launch_sweep(kites_graph *g, const uint32_t *rd, const uint32_t *U, uint32_t *chg,
                  uint32_t gate, uint32_t gate_cur) {
  sweep_args<OffT> a{(const OffT *)g->R, g->C, (const uint32_t *)g->E, g->rowid,
                     (uint32_t *)g->V, g->m, g->n, rd, U, chg, g->ctr,
                     gate, gate_cur, g->dense_edges};
  k_sweep<OP, OffT, MODE><<<g->sweep_grid, kSweepThreads, 0, g->eng->stream>>>(a);
}

// Activation of the changed rows `chg` into `wr`: the chunked push over the
// activation adjacency (rows, targets, chunk table) while the changed set is
// sparse; when `dense_pull` (vertex-level bits, vpg == 1) the pull
// activation over the in-CSC tiles takes dense changed sets.  Both are
// launched, the gate lets exactly one do the work.
template <typename OffT>
void launch_expand(kites_graph *g, const void *aR, const uint32_t *aC, const uint32_t *chunks,
                   uint64_t nchunks, bool dense_pull, uint64_t rows, uint64_t edges,
                   const uint32_t *chg, uint32_t *wr, uint32_t gate_cur, uint64_t *launches,
                   bool dense_by_next_pull = false) {
  cudaStream_t s = g->eng->stream;
  const bool sweep = dense_pull && g->rowid != nullptr;
  chunk_geom<OffT> ga{(const OffT *)aR, aC, chunks, nchunks, rows, rows + edges, g->chunk_items};
  expand_args<OffT> ea{ga, chg, wr, g->ctr, sweep ? 1u : 0u, gate_cur, g->dense_rows};
  k_expand_chunked<OffT><<<g->expand_grid, kBlock, 0, s>>>(ea);
  ++*launches;
  // A dense changed set is left to the next iteration's k_sweep_changed.
  if (sweep && !dense_by_next_pull) {
    sweep_args<OffT> sa{(const OffT *)g->R, g->C, nullptr, g->rowid, nullptr, g->m, g->n,
                        nullptr, chg, wr, g->ctr, 2u, gate_cur, g->dense_rows};
    k_activate_sweep<OffT><<<g->sweep_grid, kSweepThreads, 0, s>>>(sa);
    ++*launches;
  }
}

// One iteration of the plain strategy: pull, activation, clear, check.
// Bitmaps of parity p: frontier[p] is read (F_t), changed[p] written (U_t),
// activation writes frontier[p^1].  With edge sweeps (vpg == 1) a dense
// changed set is not expanded: the next iteration's k_sweep_changed finds
// its rows from U_t itself, so U_t (changed[p]) is kept one iteration
// longer and cleared at the end of the next one.
template <int OP, typename OffT>
int launch_iteration(kites_graph *g, int parity, cudaGraphConditionalHandle h,
                     int has_handle, uint64_t *launches, bool time_pull) {
  cudaStream_t s = g->eng->stream;
  if (time_pull) KITES_CUDA_TRY(cudaEventRecord(g->eng->kev0, s));
  chunk_geom<OffT> gin{(const OffT *)g->R, g->C, g->chunk_in, g->nchunks_in,
                       g->n, g->n + g->m, g->chunk_items};
  // Three pulls are launched and the gates let exactly one work: after a
  // dense changed set, k_sweep_changed; else on a sparse frontier the
  // per-row chunked pull, on a dense one (activation edges of the previous
  // iteration above dense_edges) the edge sweep.
  const bool sweep = g->rowid != nullptr;
  pull_args<OffT> pa{gin, (const uint32_t *)g->E, (uint32_t *)g->V,
                     g->frontier[parity], g->changed[parity], g->shift, g->ctr, nullptr,
                     sweep ? 1u : 0u, 0u, g->dense_edges, sweep ? g->dense_rows : 0ull};
  k_pull_chunked<OP, OffT><<<g->pull_grid, kBlock, 0, s>>>(pa);
  if (sweep) {
    launch_sweep<OP, OffT, kRowFilter>(g, g->frontier[parity], nullptr, g->changed[parity],
                                       2u, 0u);
    sweep_args<OffT> fa{(const OffT *)g->R, g->C, (const uint32_t *)g->E, g->rowid,
                        (uint32_t *)g->V, g->m, g->n, nullptr, g->changed[parity ^ 1],
                        g->changed[parity], g->ctr, 0u, 0u, g->dense_rows,
                        g->frontier[parity]};
    k_sweep_changed<OP, OffT><<<g->sweep_grid, kSweepThreads, 0, s>>>(fa);
    *launches += 2;
  }
  if (time_pull) KITES_CUDA_TRY(cudaEventRecord(g->eng->kev1, s));
  launch_expand<OffT>(g, g->dirR, g->dirC, g->chunk_dir, g->nchunks_dir, g->vpg == 1,
                      g->n_dir_rows, g->n_dir_edges, g->changed[parity],
                      g->frontier[parity ^ 1], 1u, launches, sweep);
  // Clear the read frontier and, with sweeps, the previous changed set;
  // without them this iteration's (adjacent words).
  if (sweep)
    k_clear_two<<<grid_for(g->nwords, 256, 4096), 256, 0, s>>>(g->frontier[parity],
                                                                g->changed[parity ^ 1], g->nwords);
  else
    k_clear_words<<<grid_for(2 * g->nwords, 256, 4096), 256, 0, s>>>(g->frontier[parity],
                                                                      2 * g->nwords);
  iter_record rec{g->rec_active, g->rec_edges, KITES_MAX_RECORDED_ITERS};
  k_loop_check<<<1, 1, 0, s>>>(g->ctr, rec, h, has_handle);
  KITES_CUDA_TRY(cudaGetLastError());
  *launches += 3;
  return KITES_OK;
}

// Batched iteration: K-wide pull over the V x K array, vertex-level
// activation, clear, check.  bits = [f0 | c0 | f1 | c1], nwords each.
struct batch_state {
  uint32_t *D;
  uint32_t *bits;
  uint64_t nwords;
  const void *actR;
  const uint32_t *actC;
  const uint32_t *act_chunks;
  uint64_t act_nchunks, act_rows, act_edges;
  int grid;
  bool tma;       // TMA row gathers (g->dmap describes D)
  int tma_grid;
  bool async;     // row gathers as cp.async copies into shared memory
  int async_grid;
};

// Grid of k_pull_batch_async: as many CTAs as its shared memory and
// registers let reside, capped by the chunk count.
template <int OP, typename OffT, int K, bool kMasked = false>
int size_async_pull(kites_graph *g, int *out) {
  const int smem = (int)async_batch_smem_bytes();
  KITES_CUDA_TRY(cudaFuncSetAttribute(k_pull_batch_async<OP, OffT, K, kMasked>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int per_sm = 0;
  KITES_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, k_pull_batch_async<OP, OffT, K, kMasked>, kBlock, smem));
  const uint64_t cap = (uint64_t)std::max(per_sm, 1) * g->eng->sm_count;
  const uint64_t want = (g->nchunks_batch + kWarpsPerBlock - 1) / kWarpsPerBlock;
  *out = (int)std::max<uint64_t>(1, std::min(want, cap));
  return KITES_OK;
}

template <int OP, typename OffT, int K>
int launch_batch_iteration(kites_graph *g, const batch_state &b, int parity,
                           cudaGraphConditionalHandle h, int has_handle, uint64_t *launches,
                           bool time_pull) {
  cudaStream_t s = g->eng->stream;
  uint32_t *rd = b.bits + (parity ? 2 : 0) * b.nwords;
  uint32_t *chg = rd + b.nwords;
  uint32_t *wr = b.bits + (parity ? 0 : 2) * b.nwords;
  if (time_pull) KITES_CUDA_TRY(cudaEventRecord(g->eng->kev0, s));
  chunk_geom<OffT> gb{(const OffT *)g->R, g->C, g->chunk_batch, g->nchunks_batch,
                      g->n, g->n + g->m, g->batch_chunk_items};
  bool launched = false;
  if constexpr (K >= 32) {
    if (b.tma) {
      tma_batch_args<OffT> ta{gb, (const uint32_t *)g->E, b.D, rd, chg, g->ctr};
      k_pull_batch_tma<OP, OffT, K><<<b.tma_grid, kTmaWarps * 32,
                                      tma_batch_smem_bytes<K, OffT>(), s>>>(g->dmap, ta);
      launched = true;
    }
  }
  if (!launched) {
    pull_batch_args<OffT> pa{gb, (const uint32_t *)g->E, b.D, rd, chg, g->ctr};
    if (b.async)
      k_pull_batch_async<OP, OffT, K><<<b.async_grid, kBlock, async_batch_smem_bytes(), s>>>(pa);
    else
      k_pull_batch<OP, OffT, K><<<b.grid, kBlock, 0, s>>>(pa);
  }
  if (time_pull) KITES_CUDA_TRY(cudaEventRecord(g->eng->kev1, s));
  launch_expand<OffT>(g, b.actR, b.actC, b.act_chunks, b.act_nchunks, true, b.act_rows,
                      b.act_edges, chg, wr, 1u, launches);
  k_clear_words<<<grid_for(2 * b.nwords, 256, 4096), 256, 0, s>>>(rd, 2 * b.nwords);
  iter_record rec{g->rec_active, g->rec_edges, KITES_MAX_RECORDED_ITERS};
  k_loop_check<<<1, 1, 0, s>>>(g->ctr, rec, h, has_handle);
  KITES_CUDA_TRY(cudaGetLastError());
  *launches += 3;
  return KITES_OK;
}

// Iterates to the fixed point.  `launch(parity, handle, has_handle,
// &launches, time_pull)` enqueues one iteration.  Device loop: a CUDA graph
// whose conditional while node runs two iterations per trip and stops when
// k_loop_check clears the condition; it is captured once per loop key and
// reused.  Host loop: one counter read-back per iteration, as
// compute.cuh:57-128 does; with time_kernels it also times each pull.
template <class Launch>
int drive_loop(kites_graph *g, const kites_run_opts &o, loop_key key, Launch launch,
               run_counters *out, float *ms, uint64_t *launches, kites_run_stats *st) {
  kites_engine *eng = g->eng;
  cudaStream_t s = eng->stream;
  run_counters init = {};
  // A monotone program reaches its fixed point within n + 1 rounds; the
  // default cap only ends a loop that cannot converge (e.g. a wrapping add
  // from 0xFFFFFFFF), with KITES_ERR_TIMEOUT.
  init.max_iterations = o.max_iterations ? o.max_iterations : 2 * g->n + 16;
  run_counters *hctr = (run_counters *)eng->pinned;
  *hctr = init;
  KITES_CUDA_TRY(cudaMemcpyAsync(g->ctr, hctr, sizeof(run_counters),
                                 cudaMemcpyHostToDevice, s));
  *launches = 0;
  const bool dev_loop = o.device_loop && !o.time_kernels;
  if (dev_loop) {
    auto it = g->loops.find(key);
    if (it == g->loops.end()) {
      cudaGraph_t graph;
      KITES_CUDA_TRY(cudaGraphCreate(&graph, 0));
      cudaGraphConditionalHandle handle;
      KITES_CUDA_TRY(cudaGraphConditionalHandleCreate(&handle, graph, 1,
                                                      cudaGraphCondAssignDefault));
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = handle;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t node;
      KITES_CUDA_TRY(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      KITES_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeThreadLocal));
      uint64_t dummy = 0;
      int st2 = launch(0, handle, 1, &dummy, false);
      if (st2 == KITES_OK) st2 = launch(1, handle, 1, &dummy, false);
      cudaGraph_t captured;
      cudaError_t e = cudaStreamEndCapture(s, &captured);
      if (st2 != KITES_OK) {
        cudaGraphDestroy(graph);
        return st2;
      }
      KITES_CUDA_TRY(e);
      cudaGraphExec_t ex;
      KITES_CUDA_TRY(cudaGraphInstantiate(&ex, graph, 0));
      it = g->loops.emplace(key, std::make_pair(graph, ex)).first;
    }
    KITES_CUDA_TRY(cudaEventRecord(eng->ev0, s));
    KITES_CUDA_TRY(cudaGraphLaunch(it->second.second, s));
  } else {
    KITES_CUDA_TRY(cudaEventRecord(eng->ev0, s));
    g->pull_log.clear();
    // The sweeps' gates read the previous iteration's activation edges and
    // changed rows.
    unsigned long long prev_out_edges = 0, prev_changed = 0;
    for (uint64_t i = 0;; ++i) {
      KITES_TRY(launch((int)(i & 1), 0, 0, launches, o.time_kernels != 0));
      KITES_CUDA_TRY(cudaMemcpyAsync(hctr, g->ctr, sizeof(run_counters),
                                     cudaMemcpyDeviceToHost, s));
      KITES_CUDA_TRY(cudaStreamSynchronize(s));
      if (o.time_kernels && st) {
        float kms = 0.f;
        KITES_CUDA_TRY(cudaEventElapsedTime(&kms, eng->kev0, eng->kev1));
        st->pull_kernel_ms += kms;
        st->pull_kernel_launches += 1;
        if (i < KITES_MAX_RECORDED_ITERS) st->iter_ms[i] = kms;
        const bool fused = g->rowid && prev_changed > g->dense_rows;
        g->pull_log.push_back({kms, fused || prev_out_edges > g->dense_edges, fused,
                               hctr->last_active, hctr->last_edges, hctr->total_updated});
      }
      prev_out_edges = hctr->last_out_edges;
      prev_changed = hctr->last_changed;
      if (hctr->done) break;
    }
  }
  KITES_CUDA_TRY(cudaEventRecord(eng->ev1, s));
  KITES_CUDA_TRY(cudaMemcpyAsync(hctr, g->ctr, sizeof(run_counters),
                                 cudaMemcpyDeviceToHost, s));
  KITES_CUDA_TRY(cudaStreamSynchronize(s));
  KITES_CUDA_TRY(cudaEventElapsedTime(ms, eng->ev0, eng->ev1));
  if (dev_loop) *launches = 4 * hctr->iterations;  // kernels that did work
  *out = *hctr;
  return KITES_OK;
}

int record_iterations(kites_graph *g, const run_counters &c, int strategy,
                      kites_run_stats *st) {
  const uint32_t nrec =
      (uint32_t)std::min<unsigned long long>(c.iterations, KITES_MAX_RECORDED_ITERS);
  st->n_recorded = nrec;
  if (nrec) {
    KITES_CUDA_TRY(cudaMemcpy(st->iter_active, g->rec_active, nrec * 8, cudaMemcpyDeviceToHost));
    KITES_CUDA_TRY(cudaMemcpy(st->iter_edges, g->rec_edges, nrec * 8, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < nrec; ++i) st->iter_strategy[i] = (uint8_t)strategy;
  }
  return KITES_OK;
}

template <int OP, typename OffT>
int run_plain(kites_graph *g, const kites_run_opts &o, kites_run_stats *st) {
  auto t0 = std::chrono::steady_clock::now();
  run_counters c;
  float ms = 0.f;
  uint64_t launches = 0;
  auto launch = [g](int parity, cudaGraphConditionalHandle h, int hh, uint64_t *l, bool tp) {
    return launch_iteration<OP, OffT>(g, parity, h, hh, l, tp);
  };
  // Both changed sets start empty (the first iteration reads changed[1] as
  // the previous one's).
  KITES_CUDA_TRY(cudaMemsetAsync(g->changed[0], 0, g->nwords * 4, g->eng->stream));
  KITES_CUDA_TRY(cudaMemsetAsync(g->changed[1], 0, g->nwords * 4, g->eng->stream));
  KITES_TRY(drive_loop(g, o, loop_key{OP, KITES_STRATEGY_PLAIN}, launch, &c, &ms, &launches, st));
  if (st) {
    st->iterations = c.iterations;
    st->device_ms = ms;
    st->edges_traversed = c.total_edges;
    const uint64_t e_bytes = op_reads_weights<OP>() ? 4 : 0;
    // Algorithmic bytes (plain pull): per iteration 2 x 4 ceil(nbits/32) for
    // the bitmap read and reset, 12 B per active vertex, (4 + eT + vT) per
    // traversed in-edge, vT + 8 per updated row and 8 per activation edge.
    const uint64_t bitmap = 8ull * ((g->nbits + 31) / 32);
    st->algorithmic_bytes = c.iterations * bitmap + 12ull * c.total_active +
                            (8ull + e_bytes) * c.total_edges + 12ull * c.total_updated +
                            8ull * c.total_out_edges;
    st->strategy_hist[KITES_STRATEGY_PLAIN] += c.iterations;
    if (o.time_kernels) {
      // Pull kernels alone, per iteration: frontier words, 12 B per active
      // vertex (V[v], R[v], R[v+1]), (4 C + eT + 4 V[src]) per in-edge, 4 B
      // per store.  A fused iteration (k_sweep_changed) also does the
      // activation of the previous changed set in pull form: every
      // in-edge's source and its changed-set word (4 + 4 bytes for all m
      // edges) in place of the frontier words.  `pull_dense_*`: the
      // iterations whose pull ran as a dense sweep.
      const uint64_t fw = 4ull * ((g->nbits + 31) / 32);
      unsigned long long upd_before = 0;
      for (const auto &r : g->pull_log) {
        const uint64_t b = 12ull * r.active + (8ull + e_bytes) * r.edges +
                           4ull * (r.total_updated - upd_before) +
                           (r.fused ? 8ull * g->m - 4ull * r.edges : fw);
        upd_before = r.total_updated;
        st->pull_kernel_bytes += b;
        if (r.dense) {
          st->pull_dense_ms += r.ms;
          st->pull_dense_launches += 1;
          st->pull_dense_bytes += b;
        }
      }
    }
    st->kernel_launches += launches;
    if (o.record_iterations) KITES_TRY(record_iterations(g, c, KITES_STRATEGY_PLAIN, st));
  }
  if (c.error) return run_error(c.error);
  if (c.timed_out)
    return fail(KITES_ERR_TIMEOUT, "no fixed point after %llu iterations",
                (unsigned long long)c.iterations);
  if (st)
    st->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return KITES_OK;
}

template <typename OffT>
int dispatch_process(kites_graph *g, int op, const kites_run_opts &o,
                     kites_run_stats *st) {
  switch (op) {
    case OP_SSSP: return run_plain<OP_SSSP, OffT>(g, o, st);
    case OP_SSSP_WRAP: return run_plain<OP_SSSP_WRAP, OffT>(g, o, st);
    case OP_BFS: return run_plain<OP_BFS, OffT>(g, o, st);
    case OP_CC: return run_plain<OP_CC, OffT>(g, o, st);
    default: return fail(KITES_ERR_UNSUPPORTED, "operator %d has no iteration loop", op);
  }
}

template <typename OffT>
int run_pagerank(kites_graph *g, uint64_t n_real, float *out, const kites_run_opts &o,
                 kites_run_stats *st) {
  kites_engine *eng = g->eng;
  cudaStream_t s = eng->stream;
  if (g->vsize != 4) return fail(KITES_ERR_UNSUPPORTED, "PageRank needs 4-byte vertex values");
  if (!g->out_deg) return fail(KITES_ERR_UNSUPPORTED, "graph has no out-degrees");
  auto t0 = std::chrono::steady_clock::now();
  void *p;
  if (!g->pr_x) {
    KITES_TRY(graph_alloc(g, &p, g->n * 4)); g->pr_x = (float *)p;
    KITES_TRY(graph_alloc(g, &p, g->n * 4)); g->pr_y = (float *)p;
    KITES_TRY(graph_alloc(g, &p, g->n * 4)); g->pr_inv_out = (float *)p;
  }
  float *pr = (float *)g->V;
  k_pr_init<<<grid_for(g->n), 256, 0, s>>>(g->out_deg, g->n, n_real, g->pr_inv_out,
                                           g->pr_x, g->pr_y, pr);
  KITES_CUDA_TRY(cudaGetLastError());
  chunk_geom<OffT> gin{(const OffT *)g->R, g->C, g->chunk_in, g->nchunks_in,
                       g->n, g->n + g->m, g->chunk_items};
  const float base = (float)((1.0 - (double)o.damping) / (double)n_real);
  KITES_CUDA_TRY(cudaEventRecord(eng->ev0, s));
  for (uint32_t it = 0; it < o.pagerank_iterations; ++it) {
    k_pr_pull<OffT><<<g->pull_grid, kBlock, 0, s>>>(gin, g->pr_x, g->pr_y);
    k_pr_update<<<grid_for(n_real), 256, 0, s>>>(n_real, base, o.damping, g->pr_inv_out,
                                                 g->pr_x, g->pr_y, pr);
  }
  KITES_CUDA_TRY(cudaGetLastError());
  KITES_CUDA_TRY(cudaEventRecord(eng->ev1, s));
  if (out) KITES_CUDA_TRY(cudaMemcpyAsync(out, pr, n_real * 4, cudaMemcpyDefault, s));
  KITES_CUDA_TRY(cudaStreamSynchronize(s));
  float ms = 0.f;
  KITES_CUDA_TRY(cudaEventElapsedTime(&ms, eng->ev0, eng->ev1));
  if (st) {
    st->iterations = o.pagerank_iterations;
    st->device_ms = ms;
    st->edges_traversed = (uint64_t)o.pagerank_iterations * g->m;
    // Per step: C and the x[u] gather per edge, R per row, then y/inv/x/pr.
    st->algorithmic_bytes = (uint64_t)o.pagerank_iterations *
                            (8ull * g->m + (g->off64 ? 8ull : 4ull) * g->n + 20ull * n_real);
    st->strategy_hist[KITES_STRATEGY_PULL_ALL] = o.pagerank_iterations;
    st->kernel_launches = 1 + 2ull * o.pagerank_iterations;
    st->host_ms = std::chrono::duration<double, std::milli>(
                      std::chrono::steady_clock::now() - t0).count();
  }
  return KITES_OK;
}

// ---- flexible loop: one strategy per iteration -------------------------------

// A: frontier scratch; U[parity]: changed by the previous iteration,
// U[parity ^ 1]: changed by this one; Q: compacted queue for PUSH.
struct flex_state {
  uint32_t *A;
  uint32_t *U[2];
  uint32_t *Q;
};

int prepare_flex(kites_graph *g, flex_state *f) {
  if (g->vpg != 1 || !g->directed)
    return fail(KITES_ERR_UNSUPPORTED,
                "per-iteration strategies need a directed graph with vertex_per_group 1");
  if (!g->queue) {
    void *p;
    KITES_TRY(graph_alloc(g, &p, g->n * 4));
    g->queue = (uint32_t *)p;
  }
  f->A = g->frontier[0];
  f->U[0] = g->changed[0];
  f->U[1] = g->changed[1];
  f->Q = g->queue;
  return KITES_OK;
}

// Enqueues the kernels of `strategy` for one iteration: U[parity] -> U[parity^1].
template <int OP, typename OffT>
int launch_strategy(kites_graph *g, const flex_state &f, int strategy, int parity,
                    uint64_t *launches) {
  cudaStream_t s = g->eng->stream;
  uint32_t *Ucur = f.U[parity], *Unext = f.U[parity ^ 1];
  chunk_geom<OffT> gin{(const OffT *)g->R, g->C, g->chunk_in, g->nchunks_in,
                       g->n, g->n + g->m, g->chunk_items};
  chunk_geom<OffT> gdir{(const OffT *)g->dirR, g->dirC, g->chunk_dir, g->nchunks_dir,
                        g->n_dir_rows, g->n_dir_rows + g->n_dir_edges, g->chunk_items};
  const uint64_t nw = g->nwords;
  auto expand = [&]() {
    // U was marked by the previous iteration: its count is last_changed.
    launch_expand<OffT>(g, g->dirR, g->dirC, g->chunk_dir, g->nchunks_dir, g->vpg == 1,
                        g->n_dir_rows, g->n_dir_edges, Ucur, f.A, 0u, launches);
  };
  switch (strategy) {
    case KITES_STRATEGY_PLAIN: {
      expand();
      // The expansion just counted this iteration's activation edges.
      pull_args<OffT> pa{gin, (const uint32_t *)g->E, (uint32_t *)g->V, f.A, Unext, 0, g->ctr,
                         nullptr, 1u, 1u, g->dense_edges};
      k_pull_chunked<OP, OffT><<<g->pull_grid, kBlock, 0, s>>>(pa);
      launch_sweep<OP, OffT, kRowFilter>(g, f.A, nullptr, Unext, 2u, 1u);
      ++*launches;
      break;
    }
    case KITES_STRATEGY_PUSH: {
      k_compact_queue<<<grid_for(nw, 256, 2048), 256, 0, s>>>(Ucur, nw, g->out_deg, f.Q, g->ctr);
      push_args<OffT> pa{(const OffT *)g->outR, g->outC, g->outE, f.Q, (uint32_t *)g->V, Unext,
                         g->ctr};
      k_push_queue<OP, OffT><<<g->eng->sm_count * 8, kBlock, 0, s>>>(pa);
      ++*launches;
      break;
    }
    case KITES_STRATEGY_PULL_ALL: {
      launch_sweep<OP, OffT, kAllRows>(g, nullptr, nullptr, Unext, 0u, 0u);
      break;
    }
    case KITES_STRATEGY_PULL_CHANGED: {
      // The frontier's rows fold only in-edges whose source is in U.
      expand();
      pull_args<OffT> pa{gin, (const uint32_t *)g->E, (uint32_t *)g->V, f.A, Unext, 0, g->ctr,
                         Ucur, 0u, 0u, 0ull, 0ull};
      k_pull_all<OP, OffT><<<g->pull_grid, kBlock, 0, s>>>(pa);
      break;
    }
    case KITES_STRATEGY_MIP: {
      // Coarse activation through the block map, then the frontier pull.
      const mip_geom mg{g->mip, g->mip_dim, g->mip_dim / 32, g->mip_block};
      uint32_t *bchg = g->mip_blocks, *bact = g->mip_blocks + mg.row_words;
      const uint64_t top = std::max<uint64_t>(nw, mg.row_words);
      k_mip_blocks<<<grid_for(top, 256, 2048), 256, 0, s>>>(Ucur, nw, mg, bchg, bact);
      const unsigned gx = (unsigned)((mg.row_words + 255) / 256);
      const unsigned gy = (unsigned)std::min<uint64_t>(
          mg.row_words, std::max<uint64_t>(1, (uint64_t)g->eng->sm_count * 8 / gx));
      k_mip_activate<<<dim3(gx, gy), 256, 0, s>>>(mg, bchg, bact);
      k_mip_expand<<<grid_for(top, 256, 2048), 256, 0, s>>>(f.A, nw, g->n, mg, bact, bchg);
      pull_args<OffT> pa{gin, (const uint32_t *)g->E, (uint32_t *)g->V, f.A, Unext, 0, g->ctr,
                         nullptr, 0u, 0u, 0ull, 0ull};
      k_pull_chunked<OP, OffT><<<g->pull_grid, kBlock, 0, s>>>(pa);
      *launches += 3;
      break;
    }
    case KITES_STRATEGY_TPV1:
    case KITES_STRATEGY_TPV4:
    case KITES_STRATEGY_TPV8:
    case KITES_STRATEGY_TPV32: {
      expand();
      pull_tpv_args<OffT> pa{(const OffT *)g->R, g->C, (const uint32_t *)g->E,
                             (uint32_t *)g->V, f.A, Unext, nw, g->ctr};
      const unsigned grid = grid_for(nw * 32, kBlock, g->eng->sm_count * 16);
      if (strategy == KITES_STRATEGY_TPV1)
        k_pull_tpv<OP, OffT, 1><<<grid, kBlock, 0, s>>>(pa);
      else if (strategy == KITES_STRATEGY_TPV4)
        k_pull_tpv<OP, OffT, 4><<<grid, kBlock, 0, s>>>(pa);
      else if (strategy == KITES_STRATEGY_TPV8)
        k_pull_tpv<OP, OffT, 8><<<grid, kBlock, 0, s>>>(pa);
      else
        k_pull_tpv<OP, OffT, 32><<<grid, kBlock, 0, s>>>(pa);
      break;
    }
    default:
      return fail(KITES_ERR_INVALID, "unknown strategy %d", strategy);
  }
  ++*launches;
  KITES_CUDA_TRY(cudaGetLastError());
  return KITES_OK;
}

template <int OP, typename OffT>
int launch_flex_iteration(kites_graph *g, const flex_state &f, int strategy, int parity,
                          cudaGraphConditionalHandle h, int hh, uint64_t *launches,
                          bool time_pull) {
  cudaStream_t s = g->eng->stream;
  if (time_pull) KITES_CUDA_TRY(cudaEventRecord(g->eng->kev0, s));
  KITES_TRY((launch_strategy<OP, OffT>(g, f, strategy, parity, launches)));
  if (time_pull) KITES_CUDA_TRY(cudaEventRecord(g->eng->kev1, s));
  k_clear_two<<<grid_for(g->nwords, 256, 4096), 256, 0, s>>>(f.A, f.U[parity], g->nwords);
  iter_record rec{g->rec_active, g->rec_edges, KITES_MAX_RECORDED_ITERS};
  k_loop_check<<<1, 1, 0, s>>>(g->ctr, rec, h, hh);
  KITES_CUDA_TRY(cudaGetLastError());
  *launches += 2;
  return KITES_OK;
}

// Runs the graph's current values from the changed set in U[0] with one
// fixed strategy per iteration.
template <int OP, typename OffT>
int run_flex(kites_graph *g, const kites_run_opts &o, kites_run_stats *st) {
  auto t0 = std::chrono::steady_clock::now();
  flex_state f;
  KITES_TRY(prepare_flex(g, &f));
  const int strategy = o.strategy;
  run_counters c;
  float ms = 0.f;
  uint64_t launches = 0;
  auto launch = [g, &f, strategy](int parity, cudaGraphConditionalHandle h, int hh,
                                  uint64_t *l, bool tp) {
    return launch_flex_iteration<OP, OffT>(g, f, strategy, parity, h, hh, l, tp);
  };
  KITES_TRY(drive_loop(g, o, loop_key{OP, 100 + strategy}, launch, &c, &ms, &launches, st));
  if (st) {
    st->iterations = c.iterations;
    st->device_ms = ms;
    st->edges_traversed = c.total_edges;
    const uint64_t e_bytes = op_reads_weights<OP>() ? 4 : 0;
    st->algorithmic_bytes = c.iterations * 8ull * g->nwords + 12ull * c.total_active +
                            (8ull + e_bytes) * c.total_edges + 12ull * c.total_updated +
                            8ull * c.total_out_edges;
    st->strategy_hist[strategy] += c.iterations;
    st->kernel_launches += launches;
    if (o.record_iterations) KITES_TRY(record_iterations(g, c, strategy, st));
    st->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  if (c.error) return run_error(c.error);
  if (c.timed_out)
    return fail(KITES_ERR_TIMEOUT, "no fixed point after %llu iterations",
                (unsigned long long)c.iterations);
  return KITES_OK;
}

template <typename OffT>
int dispatch_flex(kites_graph *g, int op, const kites_run_opts &o, kites_run_stats *st) {
  switch (op) {
    case OP_SSSP: return run_flex<OP_SSSP, OffT>(g, o, st);
    case OP_SSSP_WRAP: return run_flex<OP_SSSP_WRAP, OffT>(g, o, st);
    case OP_BFS: return run_flex<OP_BFS, OffT>(g, o, st);
    case OP_CC: return run_flex<OP_CC, OffT>(g, o, st);
    default: return fail(KITES_ERR_UNSUPPORTED, "operator %d has no iteration loop", op);
  }
}

// ---- learned selection (AUTO) ------------------------------------------------

// Strategy of each selector class.
int class_strategy(const kites_graph *g, uint32_t cls) {
  switch (cls) {
    case 1: return KITES_STRATEGY_PUSH;
    case 2: return g->coarse_strategy;
    case 3: return g->tpv_strategy;
    default: return KITES_STRATEGY_PLAIN;
  }
}

int prepare_select(kites_graph *g) {
  void *p;
  if (!g->sacc) {
    KITES_TRY(graph_alloc(g, &p, sizeof(select_acc)));
    g->sacc = p;
    KITES_CUDA_TRY(cudaMemsetAsync(p, 0, sizeof(select_acc), g->eng->stream));
  }
  if (!g->rec_sel) {
    KITES_TRY(graph_alloc(g, &p, KITES_MAX_RECORDED_ITERS));
    g->rec_sel = (uint8_t *)p;
  }
  return KITES_OK;
}

template <typename OffT>
int launch_select(kites_graph *g, const uint32_t *U, float margin, float *feat_out,
                  uint32_t feat_cap, cudaGraphConditionalHandle h, int hh, uint64_t *launches,
                  const float *params = nullptr, const uint32_t *M = nullptr,
                  uint32_t sectors = 0) {
  select_args<OffT> a{U, g->nwords, g->out_deg, (const OffT *)g->R, g->n, g->m, g->ctr,
                      (select_acc *)g->sacc, params ? params : g->eng->sel_params,
                      logf(1.f + margin), feat_out, feat_cap, h, hh, M, sectors};
  k_select<OffT><<<grid_for(g->nwords, 256, (unsigned)g->eng->sm_count * 4), 256, 0,
                   g->eng->stream>>>(a);
  k_record_sel<<<1, 1, 0, g->eng->stream>>>(g->ctr, g->rec_sel, KITES_MAX_RECORDED_ITERS);
  *launches += 2;
  KITES_CUDA_TRY(cudaGetLastError());
  return KITES_OK;
}

// Captures fn() into `graph` after `deps`; returns the capture's leaf nodes.
template <class Fn>
int capture_into(cudaStream_t s, cudaGraph_t graph, const std::vector<cudaGraphNode_t> &deps,
                 Fn fn, std::vector<cudaGraphNode_t> *leaves) {
  KITES_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, graph, deps.empty() ? nullptr : deps.data(),
                                               nullptr, deps.size(),
                                               cudaStreamCaptureModeThreadLocal));
  int st = fn();
  if (leaves && st == KITES_OK) {
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t *d = nullptr;
    size_t nd = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &d, &nd);
    if (e == cudaSuccess) leaves->assign(d, d + nd);
    else st = fail(KITES_ERR_CUDA, "capture info: %s", cudaGetErrorString(e));
  }
  cudaGraph_t out;
  cudaError_t e = cudaStreamEndCapture(s, &out);
  if (st != KITES_OK) return st;
  KITES_CUDA_TRY(e);
  return KITES_OK;
}

// Device loop of AUTO: while(not converged) { select; switch(class) {PLAIN,
// PUSH, PULL_ALL, TPV}; clear; check } for both parities.
template <int OP, typename OffT>
int build_auto_loop(kites_graph *g, const flex_state &f, float margin, cudaGraphExec_t *exec) {
  cudaStream_t s = g->eng->stream;
  cudaGraph_t graph;
  KITES_CUDA_TRY(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle hw;
  KITES_CUDA_TRY(cudaGraphConditionalHandleCreate(&hw, graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = hw;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  cudaGraphNode_t wnode;
  KITES_CUDA_TRY(cudaGraphAddNode(&wnode, graph, nullptr, 0, &wp));
  cudaGraph_t body = wp.conditional.phGraph_out[0];
  std::vector<cudaGraphNode_t> leaves;
  uint64_t dummy = 0;
  for (int parity = 0; parity < 2; ++parity) {
    cudaGraphConditionalHandle hs;
    KITES_CUDA_TRY(cudaGraphConditionalHandleCreate(&hs, body, 0, cudaGraphCondAssignDefault));
    std::vector<cudaGraphNode_t> sel_leaves;
    KITES_TRY(capture_into(s, body, leaves, [&] {
      return launch_select<OffT>(g, f.U[parity], margin, nullptr, 0, hs, 1, &dummy);
    }, &sel_leaves));
    cudaGraphNodeParams sp = {};
    sp.type = cudaGraphNodeTypeConditional;
    sp.conditional.handle = hs;
    sp.conditional.type = cudaGraphCondTypeSwitch;
    sp.conditional.size = kClasses;
    cudaGraphNode_t snode;
    KITES_CUDA_TRY(cudaGraphAddNode(&snode, body, sel_leaves.data(), sel_leaves.size(), &sp));
    for (int c = 0; c < kClasses; ++c) {
      cudaGraph_t branch = sp.conditional.phGraph_out[c];
      const int strat = class_strategy(g, (uint32_t)c);
      KITES_TRY(capture_into(s, branch, {}, [&] {
        return launch_strategy<OP, OffT>(g, f, strat, parity, &dummy);
      }, nullptr));
    }
    KITES_TRY(capture_into(s, body, {snode}, [&]() -> int {
      k_clear_two<<<grid_for(g->nwords, 256, 4096), 256, 0, s>>>(f.A, f.U[parity], g->nwords);
      iter_record rec{g->rec_active, g->rec_edges, KITES_MAX_RECORDED_ITERS};
      k_loop_check<<<1, 1, 0, s>>>(g->ctr, rec, hw, 1);
      KITES_CUDA_TRY(cudaGetLastError());
      return KITES_OK;
    }, &leaves));
  }
  KITES_CUDA_TRY(cudaGraphInstantiate(exec, graph, 0));
  g->loops.emplace(loop_key{OP, 200}, std::make_pair(graph, *exec));
  return KITES_OK;
}

template <int OP, typename OffT>
int run_auto(kites_graph *g, const kites_run_opts &o, kites_run_stats *st) {
  kites_engine *eng = g->eng;
  cudaStream_t s = eng->stream;
  auto t0 = std::chrono::steady_clock::now();
  flex_state f;
  KITES_TRY(prepare_flex(g, &f));
  KITES_TRY(prepare_select(g));
  run_counters init = {};
  init.max_iterations = o.max_iterations ? o.max_iterations : 2 * g->n + 16;
  run_counters *hctr = (run_counters *)eng->pinned;
  *hctr = init;
  KITES_CUDA_TRY(cudaMemcpyAsync(g->ctr, hctr, sizeof(run_counters), cudaMemcpyHostToDevice, s));
  uint64_t launches = 0;
  const bool dev_loop = o.device_loop && !o.time_kernels;
  if (dev_loop) {
    // The cached loop bakes in the margin it was captured with.
    auto it = g->loops.find(loop_key{OP, 200});
    cudaGraphExec_t ex;
    if (it != g->loops.end() && g->auto_margin != o.selector_margin) {
      cudaGraphExecDestroy(it->second.second);
      cudaGraphDestroy(it->second.first);
      g->loops.erase(it);
      it = g->loops.end();
    }
    if (it == g->loops.end()) {
      KITES_TRY((build_auto_loop<OP, OffT>(g, f, o.selector_margin, &ex)));
      g->auto_margin = o.selector_margin;
    } else {
      ex = it->second.second;
    }
    KITES_CUDA_TRY(cudaEventRecord(eng->ev0, s));
    KITES_CUDA_TRY(cudaGraphLaunch(ex, s));
  } else {
    KITES_CUDA_TRY(cudaEventRecord(eng->ev0, s));
    g->pull_log.clear();
    // The sweeps' gates read the previous iteration's activation edges and
    // changed rows.
    unsigned long long prev_out_edges = 0, prev_changed = 0;
    for (uint64_t i = 0;; ++i) {
      const int parity = (int)(i & 1);
      KITES_TRY(launch_select<OffT>(g, f.U[parity], o.selector_margin, nullptr, 0, 0, 0,
                                    &launches));
      KITES_CUDA_TRY(cudaMemcpyAsync(hctr, g->ctr, sizeof(run_counters), cudaMemcpyDeviceToHost, s));
      KITES_CUDA_TRY(cudaStreamSynchronize(s));
      const int strat = class_strategy(g, hctr->sel);
      KITES_TRY((launch_flex_iteration<OP, OffT>(g, f, strat, parity, 0, 0, &launches,
                                                 o.time_kernels != 0)));
      KITES_CUDA_TRY(cudaMemcpyAsync(hctr, g->ctr, sizeof(run_counters), cudaMemcpyDeviceToHost, s));
      KITES_CUDA_TRY(cudaStreamSynchronize(s));
      if (o.time_kernels && st) {
        float kms = 0.f;
        KITES_CUDA_TRY(cudaEventElapsedTime(&kms, eng->kev0, eng->kev1));
        st->pull_kernel_ms += kms;
        st->pull_kernel_launches += 1;
        if (i < KITES_MAX_RECORDED_ITERS) st->iter_ms[i] = kms;
        const bool fused = g->rowid && prev_changed > g->dense_rows;
        g->pull_log.push_back({kms, fused || prev_out_edges > g->dense_edges, fused,
                               hctr->last_active, hctr->last_edges, hctr->total_updated});
      }
      prev_out_edges = hctr->last_out_edges;
      prev_changed = hctr->last_changed;
      if (hctr->done) break;
    }
  }
  KITES_CUDA_TRY(cudaEventRecord(eng->ev1, s));
  KITES_CUDA_TRY(cudaMemcpyAsync(hctr, g->ctr, sizeof(run_counters), cudaMemcpyDeviceToHost, s));
  KITES_CUDA_TRY(cudaStreamSynchronize(s));
  run_counters c = *hctr;
  float ms = 0.f;
  KITES_CUDA_TRY(cudaEventElapsedTime(&ms, eng->ev0, eng->ev1));
  if (st) {
    const uint32_t nrec =
        (uint32_t)std::min<unsigned long long>(c.iterations, KITES_MAX_RECORDED_ITERS);
    std::vector<uint8_t> cls(nrec);
    if (nrec)
      KITES_CUDA_TRY(cudaMemcpy(cls.data(), g->rec_sel, nrec, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < nrec; ++i) st->strategy_hist[class_strategy(g, cls[i])] += 1;
    st->iterations = c.iterations;
    st->device_ms = ms;
    st->edges_traversed = c.total_edges;
    const uint64_t e_bytes = op_reads_weights<OP>() ? 4 : 0;
    st->algorithmic_bytes = c.iterations * 8ull * g->nwords + 12ull * c.total_active +
                            (8ull + e_bytes) * c.total_edges + 12ull * c.total_updated +
                            8ull * c.total_out_edges;
    st->kernel_launches += dev_loop ? 6ull * c.iterations : launches;
    if (o.record_iterations) {
      KITES_TRY(record_iterations(g, c, KITES_STRATEGY_AUTO, st));
      for (uint32_t i = 0; i < nrec && i < st->n_recorded; ++i)
        st->iter_strategy[i] = (uint8_t)class_strategy(g, cls[i]);
    }
    st->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  if (c.error) return run_error(c.error);
  if (c.timed_out)
    return fail(KITES_ERR_TIMEOUT, "no fixed point after %llu iterations",
                (unsigned long long)c.iterations);
  return KITES_OK;
}

template <typename OffT>
int dispatch_auto(kites_graph *g, int op, const kites_run_opts &o, kites_run_stats *st) {
  switch (op) {
    case OP_SSSP: return run_auto<OP_SSSP, OffT>(g, o, st);
    case OP_SSSP_WRAP: return run_auto<OP_SSSP_WRAP, OffT>(g, o, st);
    case OP_BFS: return run_auto<OP_BFS, OffT>(g, o, st);
    case OP_CC: return run_auto<OP_CC, OffT>(g, o, st);
    default: return fail(KITES_ERR_UNSUPPORTED, "operator %d has no iteration loop", op);
  }
}

// Training data: from the state at the start of every iteration, run each
// selector class once (timed with CUDA events) and restore the state; then
// advance with PLAIN.  Returns per iteration the 12 features and the 4
// class times in ms.
template <int OP, typename OffT>
int record_classes(kites_graph *g, float *feat, float *times, uint32_t cap, uint32_t *n_out) {
  kites_engine *eng = g->eng;
  cudaStream_t s = eng->stream;
  flex_state f;
  KITES_TRY(prepare_flex(g, &f));
  KITES_TRY(prepare_select(g));
  void *p;
  KITES_TRY(dev_alloc(eng, &p, (uint64_t)cap * kFeat * 4));
  float *dfeat = (float *)p;
  KITES_TRY(dev_alloc(eng, &p, g->n * 4 + 2 * g->nwords * 4 + sizeof(run_counters)));
  uint32_t *snapV = (uint32_t *)p;
  uint32_t *snapU = snapV + g->n;
  run_counters *snapC = (run_counters *)(snapU + 2 * g->nwords);
  run_counters *hctr = (run_counters *)eng->pinned;
  *hctr = run_counters{};
  hctr->max_iterations = 2 * g->n + 16;
  KITES_CUDA_TRY(cudaMemcpyAsync(g->ctr, hctr, sizeof(run_counters), cudaMemcpyHostToDevice, s));
  uint64_t launches = 0;
  uint32_t n = 0;
  int st = KITES_OK;
  for (uint64_t i = 0; i < cap; ++i) {
    const int parity = (int)(i & 1);
    if ((st = launch_select<OffT>(g, f.U[parity], 0.f, dfeat, cap, 0, 0, &launches)) != KITES_OK)
      break;
    cudaMemcpyAsync(snapV, g->V, g->n * 4, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(snapU, f.U[0], g->nwords * 4, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(snapU + g->nwords, f.U[1], g->nwords * 4, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(snapC, g->ctr, sizeof(run_counters), cudaMemcpyDeviceToDevice, s);
    for (uint32_t c = 0; c < (uint32_t)kClasses; ++c) {
      cudaMemsetAsync(f.A, 0, g->nwords * 4, s);
      cudaEventRecord(eng->kev0, s);
      st = launch_strategy<OP, OffT>(g, f, class_strategy(g, c), parity, &launches);
      cudaEventRecord(eng->kev1, s);
      if (st != KITES_OK) break;
      cudaMemcpyAsync(g->V, snapV, g->n * 4, cudaMemcpyDeviceToDevice, s);
      cudaMemcpyAsync(f.U[0], snapU, g->nwords * 4, cudaMemcpyDeviceToDevice, s);
      cudaMemcpyAsync(f.U[1], snapU + g->nwords, g->nwords * 4, cudaMemcpyDeviceToDevice, s);
      cudaMemcpyAsync(g->ctr, snapC, sizeof(run_counters), cudaMemcpyDeviceToDevice, s);
      cudaError_t e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) { st = fail(KITES_ERR_CUDA, "record: %s", cudaGetErrorString(e)); break; }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, eng->kev0, eng->kev1);
      times[(uint64_t)n * kClasses + c] = ms;
    }
    if (st != KITES_OK) break;
    cudaMemsetAsync(f.A, 0, g->nwords * 4, s);
    if ((st = launch_flex_iteration<OP, OffT>(g, f, KITES_STRATEGY_PLAIN, parity, 0, 0, &launches,
                                              false)) != KITES_OK)
      break;
    cudaMemcpyAsync(hctr, g->ctr, sizeof(run_counters), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { st = fail(KITES_ERR_CUDA, "record: %s", cudaGetErrorString(e)); break; }
    ++n;
    if (hctr->done) break;
  }
  if (st == KITES_OK && n) {
    cudaError_t e = cudaMemcpy(feat, dfeat, (uint64_t)n * kFeat * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = fail(KITES_ERR_CUDA, "record copy: %s", cudaGetErrorString(e));
  }
  cudaFreeAsync(dfeat, s);
  cudaFreeAsync(snapV, s);
  cudaStreamSynchronize(s);
  *n_out = n;
  return st;
}

template <typename OffT>
int dispatch_record(kites_graph *g, int op, float *feat, float *times, uint32_t cap,
                    uint32_t *n_out) {
  switch (op) {
    case OP_SSSP: return record_classes<OP_SSSP, OffT>(g, feat, times, cap, n_out);
    case OP_BFS: return record_classes<OP_BFS, OffT>(g, feat, times, cap, n_out);
    case OP_CC: return record_classes<OP_CC, OffT>(g, feat, times, cap, n_out);
    default: return fail(KITES_ERR_UNSUPPORTED, "recording takes SSSP, BFS or CC");
  }
}

// ---- batched multi-source runs -------------------------------------------

void graph_release(kites_graph *g, void *p) {
  if (!p) return;
  cudaFreeAsync(p, g->eng->stream);
  auto &o = g->owned;
  o.erase(std::remove(o.begin(), o.end(), p), o.end());
}

void drop_batch_loops(kites_graph *g) {
  for (auto it = g->loops.begin(); it != g->loops.end();) {
    if (it->first.strategy >= 1000) {
      cudaGraphExecDestroy(it->second.second);
      cudaGraphDestroy(it->second.first);
      it = g->loops.erase(it);
    } else {
      ++it;
    }
  }
}

// Buffers and tables of the batched path for K sources with chunk size
// `items`; reallocating anything the captured loops point at drops them.
// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); null when the driver does not provide it.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// Describes D (n rows of K uint32) for tile::gather4 copies: box = one whole
// row (K values, 128 B .. 1 KB), row coordinates are vertex ids.  False when
// the map cannot be made (the register-load kernel is used then).
static bool encode_batch_map(kites_graph *g, uint32_t K) {
  if (g->dmap_ptr == g->batchD && g->dmap_K == K) return true;
  g->dmap_ptr = nullptr;
  const auto encode = tensor_map_encoder();
  if (!encode || K < 32 || K > 256 || g->n >= (1ull << 31)) return false;
  const cuuint64_t dims[2] = {K, g->n};
  const cuuint64_t strides[1] = {(cuuint64_t)K * 4};
  const cuuint32_t box[2] = {K, 1};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode(&g->dmap, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, g->batchD, dims,
                            strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return false;
  g->dmap_ptr = g->batchD;
  g->dmap_K = K;
  return true;
}

template <typename OffT>
int prepare_batch(kites_graph *g, uint32_t K, uint32_t items, batch_state *b) {
  kites_engine *eng = g->eng;
  void *p;
  const uint64_t need = g->n * (uint64_t)K;
  if (g->batch_cap < need) {
    drop_batch_loops(g);
    graph_release(g, g->batchD);
    KITES_TRY(graph_alloc(g, &p, need * 4));
    g->batchD = (uint32_t *)p;
    g->batch_cap = need;
  }
  if (!g->d_sources) {
    KITES_TRY(graph_alloc(g, &p, 256 * 4));
    g->d_sources = (uint32_t *)p;
  }
  if (g->batch_chunk_items != items) {
    drop_batch_loops(g);
    graph_release(g, g->chunk_batch);
    g->batch_chunk_items = items;
    const uint64_t total = g->n + g->m;
    uint64_t nc = (total + items - 1) / items;
    if (nc == 0) nc = 1;
    KITES_TRY(graph_alloc(g, &p, (nc + 1) * 4));
    g->chunk_batch = (uint32_t *)p;
    g->nchunks_batch = nc;
    k_chunk_table<OffT><<<grid_for(nc + 1), 256, 0, eng->stream>>>(
        (const OffT *)g->R, g->n, nc, items, g->chunk_batch);
    KITES_CUDA_TRY(cudaGetLastError());
  }
  if (g->vpg == 1) {
    b->bits = g->bitmaps;
    b->nwords = g->nwords;
  } else {
    if (!g->bbits) {
      g->bnwords = ((g->n + 31) / 32 + 31) / 32 * 32;
      KITES_TRY(graph_alloc(g, &p, 4 * g->bnwords * 4));
      g->bbits = (uint32_t *)p;
    }
    b->bits = g->bbits;
    b->nwords = g->bnwords;
  }
  // Vertex-level activation adjacency.
  if (!g->directed) {
    b->actR = g->R; b->actC = g->C; b->act_chunks = g->chunk_in;
    b->act_nchunks = g->nchunks_in; b->act_rows = g->n; b->act_edges = g->m;
  } else if (g->vpg == 1) {
    b->actR = g->dirR; b->actC = g->dirC; b->act_chunks = g->chunk_dir;
    b->act_nchunks = g->nchunks_dir; b->act_rows = g->n; b->act_edges = g->m;
  } else {
    if (!g->chunk_out)
      KITES_TRY(build_chunk_table<OffT>(g, (const OffT *)g->outR, g->n, g->m, &g->chunk_out,
                                        &g->nchunks_out));
    b->actR = g->outR; b->actC = g->outC; b->act_chunks = g->chunk_out;
    b->act_nchunks = g->nchunks_out; b->act_rows = g->n; b->act_edges = g->m;
  }
  b->D = g->batchD;
  b->tma = g->batch_gather == 1 && encode_batch_map(g, K);
  b->async = g->batch_gather == 2;
  return KITES_OK;
}

// Copies a batch result (n_given x K values of D) to dist_out.  Synchronous,
// or -- for kites_sssp_batch_async -- staged: D is copied on the device into
// the graph's staging buffer (after the previous staged result has left it)
// and copy_stream moves the staging buffer to dist_out while the engine
// stream is free for the next batch.
int deliver_batch(kites_graph *g, const uint32_t *D, uint32_t *dist_out, uint64_t values,
                  bool async) {
  kites_engine *eng = g->eng;
  cudaStream_t s = eng->stream;
  if (!async) {
    KITES_CUDA_TRY(cudaMemcpyAsync(dist_out, D, values * 4, cudaMemcpyDefault, s));
    KITES_CUDA_TRY(cudaStreamSynchronize(s));
    return KITES_OK;
  }
  if (g->stage_cap < values) {
    KITES_CUDA_TRY(cudaStreamWaitEvent(s, eng->copied, 0));
    KITES_CUDA_TRY(cudaStreamWaitEvent(s, eng->copied2, 0));
    graph_release(g, g->stage);
    g->stage = nullptr;
    g->stage_cap = 0;
    void *p;
    KITES_TRY(graph_alloc(g, &p, values * 4));
    g->stage = (uint32_t *)p;
    g->stage_cap = values;
  }
  KITES_CUDA_TRY(cudaStreamWaitEvent(s, eng->copied, 0));
  KITES_CUDA_TRY(cudaStreamWaitEvent(s, eng->copied2, 0));
  KITES_CUDA_TRY(cudaMemcpyAsync(g->stage, D, values * 4, cudaMemcpyDeviceToDevice, s));
  KITES_CUDA_TRY(cudaEventRecord(eng->staged, s));
  // Two halves on two streams, so that two copy engines share the transfer.
  const uint64_t half = (values / 2 + 7) / 8 * 8;
  KITES_CUDA_TRY(cudaStreamWaitEvent(eng->copy_stream, eng->staged, 0));
  KITES_CUDA_TRY(cudaMemcpyAsync(dist_out, g->stage, std::min(half, values) * 4,
                                 cudaMemcpyDefault, eng->copy_stream));
  KITES_CUDA_TRY(cudaEventRecord(eng->copied, eng->copy_stream));
  KITES_CUDA_TRY(cudaStreamWaitEvent(eng->copy_stream2, eng->staged, 0));
  if (values > half)
    KITES_CUDA_TRY(cudaMemcpyAsync(dist_out + half, g->stage + half, (values - half) * 4,
                                   cudaMemcpyDefault, eng->copy_stream2));
  KITES_CUDA_TRY(cudaEventRecord(eng->copied2, eng->copy_stream2));
  return KITES_OK;
}

template <int OP, typename OffT, int K>
int run_batch(kites_graph *g, const uint32_t *sources, uint32_t *dist_out,
              const kites_run_opts &o, kites_run_stats *st) {
  kites_engine *eng = g->eng;
  cudaStream_t s = eng->stream;
  auto t0 = std::chrono::steady_clock::now();
  batch_state b{};
  const uint32_t items = g->batch_items_req ? g->batch_items_req : 256u;
  KITES_TRY(prepare_batch<OffT>(g, K, items, &b));
  int per_sm = 0;
  KITES_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, k_pull_batch<OP, OffT, K>, kBlock, 0));
  const uint64_t cap = (uint64_t)std::max(per_sm, 1) * eng->sm_count;
  const uint64_t want = (g->nchunks_batch + kWarpsPerBlock - 1) / kWarpsPerBlock;
  b.grid = (int)std::max<uint64_t>(1, std::min(want, cap));
  if constexpr (K >= 32) {
    if (b.tma) {
      const int smem = (int)tma_batch_smem_bytes<K, OffT>();
      KITES_CUDA_TRY(cudaFuncSetAttribute(k_pull_batch_tma<OP, OffT, K>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      int tma_per_sm = 0;
      KITES_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &tma_per_sm, k_pull_batch_tma<OP, OffT, K>, kTmaWarps * 32, smem));
      const uint64_t tcap = (uint64_t)std::max(tma_per_sm, 1) * eng->sm_count;
      const uint64_t twant = (g->nchunks_batch + kTmaWarps - 1) / kTmaWarps;
      b.tma_grid = (int)std::max<uint64_t>(1, std::min(twant, tcap));
    }
  } else {
    b.tma = false;
  }
  if (b.async) KITES_TRY((size_async_pull<OP, OffT, K>(g, &b.async_grid)));
  KITES_CUDA_TRY(cudaMemcpyAsync(g->d_sources, sources, K * 4, cudaMemcpyDefault, s));
  k_fill_u32<<<grid_for(g->n * K), 256, 0, s>>>(b.D, g->n * K, kInf);
  KITES_CUDA_TRY(cudaMemsetAsync(b.bits, 0, 4 * b.nwords * 4, s));
  k_seed_batch<OffT><<<K, 256, 0, s>>>(b.D, K, g->d_sources, (const OffT *)g->outR, g->outC,
                                       b.bits);
  KITES_CUDA_TRY(cudaGetLastError());
  run_counters c;
  float ms = 0.f;
  uint64_t launches = 0;
  auto launch = [g, &b](int parity, cudaGraphConditionalHandle h, int hh, uint64_t *l, bool tp) {
    return launch_batch_iteration<OP, OffT, K>(g, b, parity, h, hh, l, tp);
  };
  KITES_TRY(drive_loop(g, o, loop_key{OP, 1000 + (int)K}, launch, &c, &ms, &launches, st));
  if (dist_out) KITES_TRY(deliver_batch(g, b.D, dist_out, g->n_given * K, g->async_out));
  if (st) {
    st->iterations = c.iterations;
    st->device_ms = ms;
    st->edges_traversed = c.total_edges;
    const uint64_t e_bytes = op_reads_weights<OP>() ? 4 : 0;
    // Batched pull: per traversed in-edge C + eT + the K-wide source row;
    // per active vertex R pair + its K-wide row read (and write if updated).
    const uint64_t bitmap = 8ull * b.nwords;
    st->algorithmic_bytes = c.iterations * bitmap + (8ull + 4ull * K) * c.total_active +
                            (4ull + e_bytes + 4ull * K) * c.total_edges +
                            (4ull * K + 8ull) * c.total_updated + 8ull * c.total_out_edges;
    if (o.time_kernels)
      st->pull_kernel_bytes = c.iterations * 4ull * b.nwords +
                              (8ull + 4ull * K) * c.total_active +
                              (4ull + e_bytes + 4ull * K) * c.total_edges +
                              4ull * K * c.total_updated;
    st->strategy_hist[KITES_STRATEGY_PLAIN] += c.iterations;
    st->kernel_launches += launches + 3;
    if (o.record_iterations) KITES_TRY(record_iterations(g, c, KITES_STRATEGY_PLAIN, st));
    st->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  if (c.error) return run_error(c.error);
  if (c.timed_out)
    return fail(KITES_ERR_TIMEOUT, "no fixed point after %llu iterations",
                (unsigned long long)c.iterations);
  return KITES_OK;
}

template <int OP, typename OffT>
int dispatch_batch_k(kites_graph *g, const uint32_t *src, uint32_t k, uint32_t *out,
                     const kites_run_opts &o, kites_run_stats *st) {
  switch (k) {
    case 16: return run_batch<OP, OffT, 16>(g, src, out, o, st);
    case 32: return run_batch<OP, OffT, 32>(g, src, out, o, st);
    case 64: return run_batch<OP, OffT, 64>(g, src, out, o, st);
    case 128: return run_batch<OP, OffT, 128>(g, src, out, o, st);
    case 256: return run_batch<OP, OffT, 256>(g, src, out, o, st);
    default: return fail(KITES_ERR_INVALID, "batch size %u is not 16, 32, 64, 128 or 256", k);
  }
}

template <typename OffT>
int dispatch_batch(kites_graph *g, int op, const uint32_t *src, uint32_t k, uint32_t *out,
                   const kites_run_opts &o, kites_run_stats *st) {
  switch (op) {
    case OP_SSSP: return dispatch_batch_k<OP_SSSP, OffT>(g, src, k, out, o, st);
    case OP_SSSP_WRAP: return dispatch_batch_k<OP_SSSP_WRAP, OffT>(g, src, k, out, o, st);
    case OP_BFS: return dispatch_batch_k<OP_BFS, OffT>(g, src, k, out, o, st);
    default: return fail(KITES_ERR_INVALID, "batched runs take SSSP, SSSP_WRAP or BFS");
  }
}

// ---- batched strategies (learned + batched) ---------------------------------
//
// The batched loop with one strategy per iteration.  Its state between
// iterations is the changed set U (vertex bits) and, per vertex, the
// sectors of its K-wide row that changed (M); every strategy turns
// (U, M) into the next (U', M'):
//   PLAIN         activation of U into the frontier A, then the K-wide pull
//                 over A with whole source rows (k_pull_batch);
//   PULL_CHANGED  the same frontier, gathering only the changed sectors of
//                 each source (k_pull_batch<masked>);
//   PULL_ALL      every row over whole source rows, no activation pass (the
//                 dense iterations' frontier is nearly every row anyway);
//   PUSH          the out-edges of U's rows relax the changed sectors of
//                 their targets with atomicMin (k_push_batch).
// AUTO lets the selector pick per iteration (k_select with the batched
// weights, then a switch node), PLAIN being the fallback class.

struct batch_flex {
  uint32_t *D;
  uint32_t *A;          // frontier scratch
  uint32_t *U[2];       // changed sets by parity
  uint32_t *M[2];       // changed sectors by parity (n words each)
  uint64_t nwords;
  const void *actR;
  const uint32_t *actC;
  const uint32_t *act_chunks;
  uint64_t act_nchunks, act_rows, act_edges;
  const void *outR;     // push: out-CSR and its chunk table
  const uint32_t *out_chunks;
  uint64_t out_nchunks;
  int pull_grid, mpull_grid, push_grid;
  int async_grid;       // batch_gather 2: grid of k_pull_batch_async, else 0
  int async_mgrid;      // the same for its masked form
  int async_push_grid;  // batch_gather 2: grid of k_push_batch_async, else 0
};

// Selector class -> batched strategy.
int batch_class_strategy(uint32_t cls) {
  switch (cls) {
    case 1: return KITES_STRATEGY_PUSH;
    case 2: return KITES_STRATEGY_PULL_ALL;
    case 3: return KITES_STRATEGY_PULL_CHANGED;
    default: return KITES_STRATEGY_PLAIN;
  }
}

template <typename OffT>
int prepare_batch_flex(kites_graph *g, uint32_t K, batch_flex *f) {
  if (g->vpg != 1)
    return fail(KITES_ERR_UNSUPPORTED, "batched strategies need vertex_per_group 1");
  batch_state b{};
  const uint32_t items = g->batch_items_req ? g->batch_items_req : 256u;
  KITES_TRY(prepare_batch<OffT>(g, K, items, &b));
  void *p;
  if (!g->bmask) {
    KITES_TRY(graph_alloc(g, &p, 2 * g->n * 4));
    g->bmask = (uint32_t *)p;
  }
  // Push walks the weighted out-CSR; for directed graphs with vpg 1 the
  // activation adjacency is that out-CSR and its chunk table is shared.
  const uint32_t *oc = nullptr;
  uint64_t onc = 0;
  if (g->dirR == g->outR) {
    oc = g->chunk_dir;
    onc = g->nchunks_dir;
  } else {
    if (!g->chunk_out)
      KITES_TRY(build_chunk_table<OffT>(g, (const OffT *)g->outR, g->n, g->m, &g->chunk_out,
                                        &g->nchunks_out));
    oc = g->chunk_out;
    onc = g->nchunks_out;
  }
  f->D = b.D;
  f->nwords = b.nwords;
  f->A = b.bits;
  f->U[0] = b.bits + b.nwords;
  f->U[1] = b.bits + 3 * b.nwords;
  f->M[0] = g->bmask;
  f->M[1] = g->bmask + g->n;
  f->actR = b.actR;
  f->actC = b.actC;
  f->act_chunks = b.act_chunks;
  f->act_nchunks = b.act_nchunks;
  f->act_rows = b.act_rows;
  f->act_edges = b.act_edges;
  f->outR = g->outR;
  f->out_chunks = oc;
  f->out_nchunks = onc;
  return KITES_OK;
}

template <int OP, typename OffT, int K>
int size_batch_flex_grids(kites_graph *g, batch_flex *f) {
  const int sms = g->eng->sm_count;
  auto grid = [&](auto kernel, uint64_t chunks, int *out) -> int {
    int per_sm = 0;
    KITES_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0));
    const uint64_t cap = (uint64_t)std::max(per_sm, 1) * sms;
    const uint64_t want = (chunks + kWarpsPerBlock - 1) / kWarpsPerBlock;
    *out = (int)std::max<uint64_t>(1, std::min(want, cap));
    return KITES_OK;
  };
  KITES_TRY(grid(k_pull_batch<OP, OffT, K, false>, g->nchunks_batch, &f->pull_grid));
  KITES_TRY(grid(k_pull_batch<OP, OffT, K, true>, g->nchunks_batch, &f->mpull_grid));
  KITES_TRY(grid(k_push_batch<OP, OffT, K>, f->out_nchunks, &f->push_grid));
  f->async_grid = f->async_mgrid = f->async_push_grid = 0;
  if (g->batch_gather == 2) {
    KITES_TRY((size_async_pull<OP, OffT, K>(g, &f->async_grid)));
    KITES_TRY((size_async_pull<OP, OffT, K, true>(g, &f->async_mgrid)));
    const int smem = (int)async_push_smem_bytes();
    KITES_CUDA_TRY(cudaFuncSetAttribute(k_push_batch_async<OP, OffT, K>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0;
    KITES_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k_push_batch_async<OP, OffT, K>, kBlock, smem));
    const uint64_t cap = (uint64_t)std::max(per_sm, 1) * sms;
    const uint64_t want = (f->out_nchunks + kWarpsPerBlock - 1) / kWarpsPerBlock;
    f->async_push_grid = (int)std::max<uint64_t>(1, std::min(want, cap));
  }
  return KITES_OK;
}

// Enqueues one iteration's strategy: (U[parity], M[parity]) -> (U[parity^1],
// M[parity^1]).
template <int OP, typename OffT, int K>
int launch_batch_strategy(kites_graph *g, const batch_flex &f, int strategy, int parity,
                          uint64_t *launches) {
  cudaStream_t s = g->eng->stream;
  uint32_t *Uc = f.U[parity], *Un = f.U[parity ^ 1];
  uint32_t *Mc = f.M[parity], *Mn = f.M[parity ^ 1];
  chunk_geom<OffT> gb{(const OffT *)g->R, g->C, g->chunk_batch, g->nchunks_batch,
                      g->n, g->n + g->m, g->batch_chunk_items};
  switch (strategy) {
    case KITES_STRATEGY_PLAIN:
    case KITES_STRATEGY_PULL_CHANGED: {
      // U was marked by the previous iteration: its count is last_changed.
      launch_expand<OffT>(g, f.actR, f.actC, f.act_chunks, f.act_nchunks, true, f.act_rows,
                          f.act_edges, Uc, f.A, 0u, launches);
      pull_batch_args<OffT> pa{gb, (const uint32_t *)g->E, f.D, f.A, Un, g->ctr, Mc, Mn};
      if (strategy == KITES_STRATEGY_PLAIN && f.async_grid)
        k_pull_batch_async<OP, OffT, K><<<f.async_grid, kBlock, async_batch_smem_bytes(), s>>>(
            pa);
      else if (strategy == KITES_STRATEGY_PLAIN)
        k_pull_batch<OP, OffT, K, false><<<f.pull_grid, kBlock, 0, s>>>(pa);
      else if (f.async_mgrid)
        k_pull_batch_async<OP, OffT, K, true>
            <<<f.async_mgrid, kBlock, async_batch_smem_bytes(), s>>>(pa);
      else
        k_pull_batch<OP, OffT, K, true><<<f.mpull_grid, kBlock, 0, s>>>(pa);
      break;
    }
    case KITES_STRATEGY_PULL_ALL: {
      // Every row over whole source rows: no activation pass, and exact
      // without the changed-sector invariant (every in-edge is folded).
      pull_batch_args<OffT> pa{gb, (const uint32_t *)g->E, f.D, nullptr, Un, g->ctr, Mc, Mn};
      if (f.async_grid)
        k_pull_batch_async<OP, OffT, K><<<f.async_grid, kBlock, async_batch_smem_bytes(), s>>>(
            pa);
      else
        k_pull_batch<OP, OffT, K, false><<<f.pull_grid, kBlock, 0, s>>>(pa);
      break;
    }
    case KITES_STRATEGY_PUSH: {
      chunk_geom<OffT> go{(const OffT *)f.outR, g->outC, f.out_chunks, f.out_nchunks,
                          g->n, g->n + g->m, g->chunk_items};
      push_batch_args<OffT> pa{go, g->outE, f.D, Uc, Mc, Un, Mn, g->ctr};
      if (f.async_push_grid)
        k_push_batch_async<OP, OffT, K>
            <<<f.async_push_grid, kBlock, async_push_smem_bytes(), s>>>(pa);
      else
        k_push_batch<OP, OffT, K><<<f.push_grid, kBlock, 0, s>>>(pa);
      break;
    }
    default:
      return fail(KITES_ERR_UNSUPPORTED, "strategy %d is not a batched strategy", strategy);
  }
  ++*launches;
  KITES_CUDA_TRY(cudaGetLastError());
  return KITES_OK;
}

// Clears what the iteration consumed (the frontier scratch, U[parity] and
// M[parity]) and runs the loop check.
int launch_batch_tail(kites_graph *g, const batch_flex &f, int parity,
                      cudaGraphConditionalHandle h, int hh, uint64_t *launches) {
  cudaStream_t s = g->eng->stream;
  k_clear_two<<<grid_for(f.nwords, 256, 4096), 256, 0, s>>>(f.A, f.U[parity], f.nwords);
  k_clear_words<<<grid_for(g->n, 256, 4096), 256, 0, s>>>(f.M[parity], g->n);
  iter_record rec{g->rec_active, g->rec_edges, KITES_MAX_RECORDED_ITERS};
  k_loop_check<<<1, 1, 0, s>>>(g->ctr, rec, h, hh);
  KITES_CUDA_TRY(cudaGetLastError());
  *launches += 3;
  return KITES_OK;
}

template <int OP, typename OffT, int K>
int launch_batch_flex_iteration(kites_graph *g, const batch_flex &f, int strategy, int parity,
                                cudaGraphConditionalHandle h, int hh, uint64_t *launches,
                                bool time_pull) {
  cudaStream_t s = g->eng->stream;
  if (time_pull) KITES_CUDA_TRY(cudaEventRecord(g->eng->kev0, s));
  KITES_TRY((launch_batch_strategy<OP, OffT, K>(g, f, strategy, parity, launches)));
  if (time_pull) KITES_CUDA_TRY(cudaEventRecord(g->eng->kev1, s));
  return launch_batch_tail(g, f, parity, h, hh, launches);
}

// Device loop of batched AUTO: while (not converged) { select; switch(class)
// {PLAIN, PUSH, PULL_ALL, PULL_CHANGED}; clear; check } for both parities.
template <int OP, typename OffT, int K>
int build_batch_auto_loop(kites_graph *g, const batch_flex &f, float margin,
                          cudaGraphExec_t *exec) {
  cudaStream_t s = g->eng->stream;
  cudaGraph_t graph;
  KITES_CUDA_TRY(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle hw;
  KITES_CUDA_TRY(cudaGraphConditionalHandleCreate(&hw, graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = hw;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  cudaGraphNode_t wnode;
  KITES_CUDA_TRY(cudaGraphAddNode(&wnode, graph, nullptr, 0, &wp));
  cudaGraph_t body = wp.conditional.phGraph_out[0];
  std::vector<cudaGraphNode_t> leaves;
  uint64_t dummy = 0;
  for (int parity = 0; parity < 2; ++parity) {
    cudaGraphConditionalHandle hs;
    KITES_CUDA_TRY(cudaGraphConditionalHandleCreate(&hs, body, 0, cudaGraphCondAssignDefault));
    std::vector<cudaGraphNode_t> sel_leaves;
    KITES_TRY(capture_into(s, body, leaves, [&] {
      return launch_select<OffT>(g, f.U[parity], margin, nullptr, 0, hs, 1, &dummy,
                                 g->eng->sel_params_batch, f.M[parity], K / 8);
    }, &sel_leaves));
    cudaGraphNodeParams sp = {};
    sp.type = cudaGraphNodeTypeConditional;
    sp.conditional.handle = hs;
    sp.conditional.type = cudaGraphCondTypeSwitch;
    sp.conditional.size = kClasses;
    cudaGraphNode_t snode;
    KITES_CUDA_TRY(cudaGraphAddNode(&snode, body, sel_leaves.data(), sel_leaves.size(), &sp));
    for (int c = 0; c < kClasses; ++c) {
      cudaGraph_t branch = sp.conditional.phGraph_out[c];
      const int strat = batch_class_strategy((uint32_t)c);
      KITES_TRY(capture_into(s, branch, {}, [&] {
        return launch_batch_strategy<OP, OffT, K>(g, f, strat, parity, &dummy);
      }, nullptr));
    }
    KITES_TRY(capture_into(s, body, {snode}, [&]() -> int {
      return launch_batch_tail(g, f, parity, hw, 1, &dummy);
    }, &leaves));
  }
  KITES_CUDA_TRY(cudaGraphInstantiate(exec, graph, 0));
  g->loops.emplace(loop_key{OP, 3000 + K}, std::make_pair(graph, *exec));
  return KITES_OK;
}

// Batched SSSP/BFS with a per-iteration strategy (o.strategy: AUTO, PUSH,
// PULL_ALL, PULL_CHANGED, or PLAIN through this loop when forced).
template <int OP, typename OffT, int K>
int run_batch_flex(kites_graph *g, const uint32_t *sources, uint32_t *dist_out,
                   const kites_run_opts &o, kites_run_stats *st) {
  kites_engine *eng = g->eng;
  cudaStream_t s = eng->stream;
  auto t0 = std::chrono::steady_clock::now();
  batch_flex f{};
  KITES_TRY(prepare_batch_flex<OffT>(g, K, &f));
  KITES_TRY((size_batch_flex_grids<OP, OffT, K>(g, &f)));
  const bool autosel = o.strategy == KITES_STRATEGY_AUTO;
  if (autosel) KITES_TRY(prepare_select(g));
  KITES_CUDA_TRY(cudaMemcpyAsync(g->d_sources, sources, K * 4, cudaMemcpyDefault, s));
  k_fill_u32<<<grid_for(g->n * K), 256, 0, s>>>(f.D, g->n * K, kInf);
  KITES_CUDA_TRY(cudaMemsetAsync(f.A, 0, 4 * f.nwords * 4, s));
  KITES_CUDA_TRY(cudaMemsetAsync(g->bmask, 0, 2 * g->n * 4, s));
  k_seed_batch_changed<<<1, 256, 0, s>>>(f.D, K, g->d_sources, f.U[0], f.M[0]);
  KITES_CUDA_TRY(cudaGetLastError());
  run_counters c;
  float ms = 0.f;
  uint64_t launches = 0;
  const bool dev_loop = o.device_loop && !o.time_kernels;
  if (autosel && dev_loop) {
    // The cached loop bakes in the margin it was captured with.
    const loop_key key{OP, 3000 + (int)K};
    auto it = g->loops.find(key);
    if (it != g->loops.end() && g->auto_margin_batch != o.selector_margin) {
      cudaGraphExecDestroy(it->second.second);
      cudaGraphDestroy(it->second.first);
      g->loops.erase(it);
      it = g->loops.end();
    }
    cudaGraphExec_t ex;
    if (it == g->loops.end()) {
      KITES_TRY((build_batch_auto_loop<OP, OffT, K>(g, f, o.selector_margin, &ex)));
      g->auto_margin_batch = o.selector_margin;
    } else {
      ex = it->second.second;
    }
    run_counters *hctr = (run_counters *)eng->pinned;
    *hctr = run_counters{};
    hctr->max_iterations = o.max_iterations ? o.max_iterations : 2 * g->n + 16;
    KITES_CUDA_TRY(cudaMemcpyAsync(g->ctr, hctr, sizeof(run_counters), cudaMemcpyHostToDevice, s));
    KITES_CUDA_TRY(cudaEventRecord(eng->ev0, s));
    KITES_CUDA_TRY(cudaGraphLaunch(ex, s));
    KITES_CUDA_TRY(cudaEventRecord(eng->ev1, s));
    KITES_CUDA_TRY(cudaMemcpyAsync(hctr, g->ctr, sizeof(run_counters), cudaMemcpyDeviceToHost, s));
    KITES_CUDA_TRY(cudaStreamSynchronize(s));
    KITES_CUDA_TRY(cudaEventElapsedTime(&ms, eng->ev0, eng->ev1));
    c = *hctr;
    launches = 6ull * c.iterations;
  } else if (autosel) {
    // Host loop: select, read the class back, run it (timed per iteration).
    run_counters *hctr = (run_counters *)eng->pinned;
    *hctr = run_counters{};
    hctr->max_iterations = o.max_iterations ? o.max_iterations : 2 * g->n + 16;
    KITES_CUDA_TRY(cudaMemcpyAsync(g->ctr, hctr, sizeof(run_counters), cudaMemcpyHostToDevice, s));
    KITES_CUDA_TRY(cudaEventRecord(eng->ev0, s));
    for (uint64_t i = 0;; ++i) {
      const int parity = (int)(i & 1);
      KITES_TRY(launch_select<OffT>(g, f.U[parity], o.selector_margin, nullptr, 0, 0, 0,
                                    &launches, eng->sel_params_batch, f.M[parity], K / 8));
      KITES_CUDA_TRY(cudaMemcpyAsync(hctr, g->ctr, sizeof(run_counters), cudaMemcpyDeviceToHost, s));
      KITES_CUDA_TRY(cudaStreamSynchronize(s));
      const int strat = batch_class_strategy(hctr->sel);
      KITES_TRY((launch_batch_flex_iteration<OP, OffT, K>(g, f, strat, parity, 0, 0, &launches,
                                                         o.time_kernels != 0)));
      KITES_CUDA_TRY(cudaMemcpyAsync(hctr, g->ctr, sizeof(run_counters), cudaMemcpyDeviceToHost, s));
      KITES_CUDA_TRY(cudaStreamSynchronize(s));
      if (o.time_kernels && st) {
        float kms = 0.f;
        KITES_CUDA_TRY(cudaEventElapsedTime(&kms, eng->kev0, eng->kev1));
        st->pull_kernel_ms += kms;
        st->pull_kernel_launches += 1;
        if (i < KITES_MAX_RECORDED_ITERS) st->iter_ms[i] = kms;
      }
      if (hctr->done) break;
    }
    KITES_CUDA_TRY(cudaEventRecord(eng->ev1, s));
    KITES_CUDA_TRY(cudaMemcpyAsync(hctr, g->ctr, sizeof(run_counters), cudaMemcpyDeviceToHost, s));
    KITES_CUDA_TRY(cudaStreamSynchronize(s));
    KITES_CUDA_TRY(cudaEventElapsedTime(&ms, eng->ev0, eng->ev1));
    c = *hctr;
  } else {
    const int strategy = o.strategy;
    auto launch = [g, &f, strategy](int parity, cudaGraphConditionalHandle h, int hh,
                                    uint64_t *l, bool tp) {
      return launch_batch_flex_iteration<OP, OffT, K>(g, f, strategy, parity, h, hh, l, tp);
    };
    KITES_TRY(drive_loop(g, o, loop_key{OP, 2000 + 16 * strategy + (int)(K / 16)}, launch, &c,
                         &ms, &launches, st));
  }
  if (dist_out) KITES_TRY(deliver_batch(g, f.D, dist_out, g->n_given * K, g->async_out));
  if (st) {
    st->iterations = c.iterations;
    st->device_ms = ms;
    st->edges_traversed = c.total_edges;
    const uint64_t e_bytes = op_reads_weights<OP>() ? 4 : 0;
    // Bytes as the unmasked pull would move them (an upper bound for the
    // masked strategies, which skip unchanged sectors).
    st->algorithmic_bytes = c.iterations * 8ull * f.nwords + (8ull + 4ull * K) * c.total_active +
                            (4ull + e_bytes + 4ull * K) * c.total_edges +
                            (4ull * K + 8ull) * c.total_updated + 8ull * c.total_out_edges;
    const uint32_t nrec =
        (uint32_t)std::min<unsigned long long>(c.iterations, KITES_MAX_RECORDED_ITERS);
    std::vector<uint8_t> cls(nrec, 0);
    if (autosel && nrec)
      KITES_CUDA_TRY(cudaMemcpy(cls.data(), g->rec_sel, nrec, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < nrec; ++i)
      st->strategy_hist[autosel ? batch_class_strategy(cls[i]) : o.strategy] += 1;
    st->kernel_launches += launches + 3;
    if (o.record_iterations) {
      KITES_TRY(record_iterations(g, c, o.strategy, st));
      for (uint32_t i = 0; i < nrec && i < st->n_recorded; ++i)
        st->iter_strategy[i] = (uint8_t)(autosel ? batch_class_strategy(cls[i]) : o.strategy);
    }
    st->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  if (c.error) return run_error(c.error);
  if (c.timed_out)
    return fail(KITES_ERR_TIMEOUT, "no fixed point after %llu iterations",
                (unsigned long long)c.iterations);
  return KITES_OK;
}

// Training data for the batched selector: from the state at the start of
// every iteration, each class runs once (timed with CUDA events) and the
// state (D, U, M, counters) is restored; then the loop advances with PLAIN.
template <int OP, typename OffT, int K>
int record_batch_classes(kites_graph *g, const uint32_t *sources, float *feat, float *times,
                         uint32_t cap, uint32_t *n_out) {
  kites_engine *eng = g->eng;
  cudaStream_t s = eng->stream;
  batch_flex f{};
  KITES_TRY(prepare_batch_flex<OffT>(g, K, &f));
  KITES_TRY((size_batch_flex_grids<OP, OffT, K>(g, &f)));
  KITES_TRY(prepare_select(g));
  KITES_CUDA_TRY(cudaMemcpyAsync(g->d_sources, sources, K * 4, cudaMemcpyDefault, s));
  k_fill_u32<<<grid_for(g->n * K), 256, 0, s>>>(f.D, g->n * K, kInf);
  KITES_CUDA_TRY(cudaMemsetAsync(f.A, 0, 4 * f.nwords * 4, s));
  KITES_CUDA_TRY(cudaMemsetAsync(g->bmask, 0, 2 * g->n * 4, s));
  k_seed_batch_changed<<<1, 256, 0, s>>>(f.D, K, g->d_sources, f.U[0], f.M[0]);
  KITES_CUDA_TRY(cudaGetLastError());
  void *p;
  KITES_TRY(dev_alloc(eng, &p, (uint64_t)cap * kFeat * 4));
  float *dfeat = (float *)p;
  const size_t dbytes = g->n * (size_t)K * 4, bbytes = 4 * f.nwords * 4, mbytes = 2 * g->n * 4;
  int st = dev_alloc(eng, &p, dbytes + bbytes + mbytes + sizeof(run_counters));
  if (st != KITES_OK) {
    cudaFreeAsync(dfeat, s);
    return st;
  }
  uint8_t *snap = (uint8_t *)p;
  run_counters *snapC = (run_counters *)(snap + dbytes + bbytes + mbytes);
  run_counters *hctr = (run_counters *)eng->pinned;
  *hctr = run_counters{};
  hctr->max_iterations = 2 * g->n + 16;
  cudaMemcpyAsync(g->ctr, hctr, sizeof(run_counters), cudaMemcpyHostToDevice, s);
  auto save = [&](bool restore) {
    auto cp = [&](void *a, void *b, size_t n) {
      if (restore) cudaMemcpyAsync(a, b, n, cudaMemcpyDeviceToDevice, s);
      else cudaMemcpyAsync(b, a, n, cudaMemcpyDeviceToDevice, s);
    };
    cp(f.D, snap, dbytes);
    cp(f.A, snap + dbytes, bbytes);
    cp(g->bmask, snap + dbytes + bbytes, mbytes);
    cp(g->ctr, snapC, sizeof(run_counters));
  };
  uint64_t launches = 0;
  uint32_t n = 0;
  for (uint64_t i = 0; i < cap; ++i) {
    const int parity = (int)(i & 1);
    if ((st = launch_select<OffT>(g, f.U[parity], 0.f, dfeat, cap, 0, 0, &launches,
                                  eng->sel_params_batch, f.M[parity], K / 8)) != KITES_OK)
      break;
    save(false);
    for (uint32_t c = 0; c < (uint32_t)kClasses; ++c) {
      cudaEventRecord(eng->kev0, s);
      st = launch_batch_strategy<OP, OffT, K>(g, f, batch_class_strategy(c), parity, &launches);
      cudaEventRecord(eng->kev1, s);
      if (st != KITES_OK) break;
      save(true);
      cudaError_t e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) { st = fail(KITES_ERR_CUDA, "record: %s", cudaGetErrorString(e)); break; }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, eng->kev0, eng->kev1);
      times[(uint64_t)n * kClasses + c] = ms;
    }
    if (st != KITES_OK) break;
    if ((st = launch_batch_flex_iteration<OP, OffT, K>(g, f, KITES_STRATEGY_PLAIN, parity, 0, 0,
                                                       &launches, false)) != KITES_OK)
      break;
    cudaMemcpyAsync(hctr, g->ctr, sizeof(run_counters), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { st = fail(KITES_ERR_CUDA, "record: %s", cudaGetErrorString(e)); break; }
    ++n;
    if (hctr->done) break;
  }
  if (st == KITES_OK && n) {
    cudaError_t e = cudaMemcpy(feat, dfeat, (uint64_t)n * kFeat * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = fail(KITES_ERR_CUDA, "record copy: %s", cudaGetErrorString(e));
  }
  cudaFreeAsync(dfeat, s);
  cudaFreeAsync(snap, s);
  cudaStreamSynchronize(s);
  *n_out = n;
  return st;
}

template <int OP, typename OffT>
int dispatch_batch_flex_k(kites_graph *g, const uint32_t *src, uint32_t k, uint32_t *out,
                          const kites_run_opts &o, kites_run_stats *st) {
  switch (k) {
    case 16: return run_batch_flex<OP, OffT, 16>(g, src, out, o, st);
    case 32: return run_batch_flex<OP, OffT, 32>(g, src, out, o, st);
    case 64: return run_batch_flex<OP, OffT, 64>(g, src, out, o, st);
    case 128: return run_batch_flex<OP, OffT, 128>(g, src, out, o, st);
    case 256: return run_batch_flex<OP, OffT, 256>(g, src, out, o, st);
    default: return fail(KITES_ERR_INVALID, "batch size %u is not 16, 32, 64, 128 or 256", k);
  }
}

template <typename OffT>
int dispatch_batch_flex(kites_graph *g, int op, const uint32_t *src, uint32_t k, uint32_t *out,
                        const kites_run_opts &o, kites_run_stats *st) {
  switch (op) {
    case OP_SSSP: return dispatch_batch_flex_k<OP_SSSP, OffT>(g, src, k, out, o, st);
    case OP_BFS: return dispatch_batch_flex_k<OP_BFS, OffT>(g, src, k, out, o, st);
    default:
      return fail(KITES_ERR_UNSUPPORTED,
                  "batched strategies other than PLAIN take the saturating SSSP or BFS");
  }
}

template <int OP, typename OffT>
int dispatch_record_batch_k(kites_graph *g, const uint32_t *src, uint32_t k, float *feat,
                            float *times, uint32_t cap, uint32_t *n_out) {
  switch (k) {
    case 16: return record_batch_classes<OP, OffT, 16>(g, src, feat, times, cap, n_out);
    case 32: return record_batch_classes<OP, OffT, 32>(g, src, feat, times, cap, n_out);
    case 64: return record_batch_classes<OP, OffT, 64>(g, src, feat, times, cap, n_out);
    case 128: return record_batch_classes<OP, OffT, 128>(g, src, feat, times, cap, n_out);
    case 256: return record_batch_classes<OP, OffT, 256>(g, src, feat, times, cap, n_out);
    default: return fail(KITES_ERR_INVALID, "batch size %u is not 16, 32, 64, 128 or 256", k);
  }
}

int check_graph(kites_engine *eng, kites_graph *g) {
  if (!eng || !g) return fail(KITES_ERR_INVALID, "null engine or graph");
  if (g->eng != eng) return fail(KITES_ERR_INVALID, "graph belongs to another engine");
  return set_device(eng);
}

// AUTO's fallback margins when the caller leaves selector_margin negative:
// the single-source selector's classes differ by large factors and a wrong
// pick is costly; the batched selector's differ by a few per cent in the
// dense iterations (the pull over every row against PLAIN), and at R-MAT
// scale 24 margins 0 to 0.05 ran 256.5-256.7 GTEPS against 242.4 at 0.1.
constexpr float kSelectorMargin = 0.1f;
constexpr float kSelectorMarginBatch = 0.03f;

kites_run_opts resolve_opts(const kites_run_opts *opts, bool batched = false) {
  kites_run_opts o;
  kites_default_run_opts(&o);
  if (opts) o = *opts;
  if (o.selector_margin < 0.f) o.selector_margin = batched ? kSelectorMarginBatch : kSelectorMargin;
  if (o.pagerank_iterations == 0) o.pagerank_iterations = 20;
  if (o.damping <= 0.f) o.damping = 0.85f;
  return o;
}

}  // namespace
}  // namespace kites_internal

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" const char *kites_last_error_string(void) { return error_buffer(); }

extern "C" int kites_abi_version(void) { return KITES_B200_ABI_VERSION; }

extern "C" void kites_default_run_opts(kites_run_opts *o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->strategy = KITES_STRATEGY_PLAIN;
  o->device_loop = 1;
  o->pagerank_iterations = 20;
  o->damping = 0.85f;
  o->selector_margin = -1.f;   // negative: the loop's own default (resolve_opts)
}

extern "C" int kites_engine_create(int device, kites_engine **out) {
  clear_error();
  if (!out) return fail(KITES_ERR_INVALID, "null output");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(KITES_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
  }
  if (device < 0 || device >= count)
    return fail(KITES_ERR_INVALID, "device %d out of range (%d devices)", device, count);
  cudaDeviceProp prop;
  KITES_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return fail(KITES_ERR_NO_DEVICE, "device %d is sm_%d%d; this build targets sm_100a",
                device, prop.major, prop.minor);
  KITES_CUDA_TRY(cudaSetDevice(device));
  kites_engine *eng = new kites_engine();
  eng->device = device;
  eng->sm_count = prop.multiProcessorCount;
  eng->l2_bytes = prop.l2CacheSize;
  int st = KITES_OK;
  do {
    cudaError_t ce;
    if ((ce = cudaStreamCreateWithFlags(&eng->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (ce = cudaEventCreate(&eng->ev0)) != cudaSuccess ||
        (ce = cudaEventCreate(&eng->ev1)) != cudaSuccess ||
        (ce = cudaEventCreate(&eng->kev0)) != cudaSuccess ||
        (ce = cudaEventCreate(&eng->kev1)) != cudaSuccess ||
        (ce = cudaStreamCreateWithFlags(&eng->copy_stream, cudaStreamNonBlocking)) !=
            cudaSuccess ||
        (ce = cudaStreamCreateWithFlags(&eng->copy_stream2, cudaStreamNonBlocking)) !=
            cudaSuccess ||
        (ce = cudaEventCreateWithFlags(&eng->staged, cudaEventDisableTiming)) != cudaSuccess ||
        (ce = cudaEventCreateWithFlags(&eng->copied, cudaEventDisableTiming)) != cudaSuccess ||
        (ce = cudaEventCreateWithFlags(&eng->copied2, cudaEventDisableTiming)) != cudaSuccess) {
      st = fail(KITES_ERR_CUDA, "stream/event creation failed: %s", cudaGetErrorString(ce));
      break;
    }
    cudaMemPoolProps pp = {};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = device;
    if ((ce = cudaMemPoolCreate(&eng->pool, &pp)) != cudaSuccess) {
      st = fail(KITES_ERR_CUDA, "memory pool creation failed: %s", cudaGetErrorString(ce));
      break;
    }
    uint64_t keep = ~0ull;  // never give reserved memory back between calls
    cudaMemPoolSetAttribute(eng->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if ((ce = cudaHostAlloc(&eng->pinned, 4096, cudaHostAllocPortable)) != cudaSuccess) {
      st = fail(KITES_ERR_OOM, "pinned scratch allocation failed: %s", cudaGetErrorString(ce));
      break;
    }
    if ((ce = cudaMalloc((void **)&eng->sel_params, kParams * sizeof(float))) != cudaSuccess) {
      st = fail(KITES_ERR_OOM, "selector allocation failed: %s", cudaGetErrorString(ce));
      break;
    }
#ifdef KITES_HAVE_DEFAULT_SELECTOR
    ce = cudaMemcpyAsync(eng->sel_params, kDefaultSelector, sizeof(kDefaultSelector),
                         cudaMemcpyHostToDevice, eng->stream);
    if (ce != cudaSuccess) {
      st = fail(KITES_ERR_CUDA, "selector init failed: %s", cudaGetErrorString(ce));
      break;
    }
#else
    k_mlp_neutral<<<1, 256, 0, eng->stream>>>(eng->sel_params);
#endif
    if ((ce = cudaMalloc((void **)&eng->sel_params_batch, kParams * sizeof(float))) !=
        cudaSuccess) {
      st = fail(KITES_ERR_OOM, "selector allocation failed: %s", cudaGetErrorString(ce));
      break;
    }
#ifdef KITES_HAVE_DEFAULT_BATCH_SELECTOR
    ce = cudaMemcpyAsync(eng->sel_params_batch, kDefaultBatchSelector,
                         sizeof(kDefaultBatchSelector), cudaMemcpyHostToDevice, eng->stream);
    if (ce != cudaSuccess) {
      st = fail(KITES_ERR_CUDA, "selector init failed: %s", cudaGetErrorString(ce));
      break;
    }
#else
    k_mlp_neutral<<<1, 256, 0, eng->stream>>>(eng->sel_params_batch);
#endif
    if ((ce = cudaStreamSynchronize(eng->stream)) != cudaSuccess) {
      st = fail(KITES_ERR_CUDA, "selector init failed: %s", cudaGetErrorString(ce));
      break;
    }
  } while (0);
  if (st != KITES_OK) {
    kites_engine_destroy(eng);
    return st;
  }
  *out = eng;
  return KITES_OK;
}

extern "C" int kites_engine_destroy(kites_engine *eng) {
  if (!eng) return KITES_OK;
  cudaSetDevice(eng->device);
  if (eng->stream) cudaStreamSynchronize(eng->stream);
  if (eng->copy_stream) cudaStreamSynchronize(eng->copy_stream);
  if (eng->copy_stream2) cudaStreamSynchronize(eng->copy_stream2);
  // Graphs die with their engine; their handles are invalid afterwards.
  while (!eng->graphs.empty()) kites_graph_destroy(eng->graphs.back());
  if (eng->pinned) cudaFreeHost(eng->pinned);
  if (eng->sel_params) cudaFree(eng->sel_params);
  if (eng->sel_params_batch) cudaFree(eng->sel_params_batch);
  if (eng->ev0) cudaEventDestroy(eng->ev0);
  if (eng->ev1) cudaEventDestroy(eng->ev1);
  if (eng->kev0) cudaEventDestroy(eng->kev0);
  if (eng->kev1) cudaEventDestroy(eng->kev1);
  if (eng->staged) cudaEventDestroy(eng->staged);
  if (eng->copied) cudaEventDestroy(eng->copied);
  if (eng->copied2) cudaEventDestroy(eng->copied2);
  if (eng->copy_stream) cudaStreamDestroy(eng->copy_stream);
  if (eng->copy_stream2) cudaStreamDestroy(eng->copy_stream2);
  if (eng->stream) cudaStreamDestroy(eng->stream);
  if (eng->pool) cudaMemPoolDestroy(eng->pool);
  delete eng;
  return KITES_OK;
}

extern "C" int kites_engine_mem_usage(kites_engine *eng, uint64_t *used,
                                      uint64_t *total, uint64_t *pool_reserved) {
  clear_error();
  if (!eng) return fail(KITES_ERR_INVALID, "null engine");
  KITES_TRY(set_device(eng));
  size_t fr = 0, tot = 0;
  KITES_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
  if (used) *used = tot - fr;
  if (total) *total = tot;
  if (pool_reserved) {
    uint64_t r = 0;
    KITES_CUDA_TRY(cudaMemPoolGetAttribute(eng->pool, cudaMemPoolAttrReservedMemCurrent, &r));
    *pool_reserved = r;
  }
  return KITES_OK;
}

extern "C" int kites_engine_stream(kites_engine *eng, void **stream_out) {
  clear_error();
  if (!eng || !stream_out) return fail(KITES_ERR_INVALID, "null argument");
  *stream_out = (void *)eng->stream;
  return KITES_OK;
}

extern "C" int kites_engine_sync(kites_engine *eng) {
  clear_error();
  if (!eng) return fail(KITES_ERR_INVALID, "null engine");
  KITES_TRY(set_device(eng));
  KITES_CUDA_TRY(cudaStreamSynchronize(eng->stream));
  KITES_CUDA_TRY(cudaStreamSynchronize(eng->copy_stream));
  KITES_CUDA_TRY(cudaStreamSynchronize(eng->copy_stream2));
  return KITES_OK;
}

extern "C" int kites_engine_join(kites_engine *eng) {
  clear_error();
  if (!eng) return fail(KITES_ERR_INVALID, "null engine");
  KITES_TRY(set_device(eng));
  KITES_CUDA_TRY(cudaEventRecord(eng->copied, eng->copy_stream));
  KITES_CUDA_TRY(cudaEventRecord(eng->copied2, eng->copy_stream2));
  KITES_CUDA_TRY(cudaStreamWaitEvent(eng->stream, eng->copied, 0));
  KITES_CUDA_TRY(cudaStreamWaitEvent(eng->stream, eng->copied2, 0));
  return KITES_OK;
}

extern "C" int kites_graph_destroy(kites_graph *g) {
  if (!g) return KITES_OK;
  cudaSetDevice(g->eng->device);
  cudaStreamSynchronize(g->eng->copy_stream);
  cudaStreamSynchronize(g->eng->copy_stream2);
  cudaStreamSynchronize(g->eng->stream);
  for (auto &kv : g->loops) {
    cudaGraphExecDestroy(kv.second.second);
    cudaGraphDestroy(kv.second.first);
  }
  for (void *p : g->owned) cudaFreeAsync(p, g->eng->stream);
  cudaStreamSynchronize(g->eng->stream);
  auto &live = g->eng->graphs;
  live.erase(std::remove(live.begin(), live.end(), g), live.end());
  delete g;
  return KITES_OK;
}

extern "C" int kites_graph_upload(kites_engine *eng, const kites_csc_view *v,
                                  kites_graph **out) {
  clear_error();
  if (!eng || !v || !out) return fail(KITES_ERR_INVALID, "null argument");
  *out = nullptr;
  if (v->n_vertices == 0) return fail(KITES_ERR_INVALID, "graph has no vertices");
  if (v->n_vertices >= 0xFFFFFF00ull)
    return fail(KITES_ERR_INVALID, "vertex ids must fit in 32 bits");
  if (!v->row_offsets && !v->row_offsets32)
    return fail(KITES_ERR_INVALID, "no row offsets");
  if (v->n_edges && !v->col_indices) return fail(KITES_ERR_INVALID, "no column indices");
  if (v->row_offsets32 && v->n_edges > 0xFFFFFFFFull)
    return fail(KITES_ERR_INVALID, "32-bit offsets with >= 2^32 edges");
  const uint32_t vpg = v->vertex_per_group ? v->vertex_per_group : 1;
  if (vpg & (vpg - 1)) return fail(KITES_ERR_INVALID, "vertex_per_group %u is not a power of two", vpg);
  if (v->edge_value_size && !v->edge_values && v->n_edges)
    return fail(KITES_ERR_INVALID, "edge_value_size set but no edge values");
  KITES_TRY(set_device(eng));
  kites_graph *g = new kites_graph();
  g->eng = eng;
  eng->graphs.push_back(g);
  g->n_given = v->n_vertices;
  g->n = (v->n_vertices + 127) / 128 * 128;
  g->m = v->n_edges;
  g->vpg = vpg;
  while ((1u << g->shift) < vpg) ++g->shift;
  g->directed = v->directed ? 1 : 0;
  g->off64 = v->offsets64 != 0 || g->m > 0xFFFFFFFFull - g->n;
  g->vsize = v->vertex_value_size ? v->vertex_value_size : 4;
  g->esize = v->edge_value_size;
  int st = g->off64 ? upload_typed<uint64_t>(g, v) : upload_typed<uint32_t>(g, v);
  void *p = nullptr;
  if (st == KITES_OK) {
    g->nbits = (g->n + vpg - 1) / vpg;
    g->nwords = ((g->nbits + 31) / 32 + 31) / 32 * 32;  // 128-B aligned rows
    st = graph_alloc(g, &p, 4 * g->nwords * 4);
  }
  if (st == KITES_OK) {
    g->bitmaps = (uint32_t *)p;
    g->frontier[0] = g->bitmaps;
    g->changed[0] = g->bitmaps + g->nwords;
    g->frontier[1] = g->bitmaps + 2 * g->nwords;
    g->changed[1] = g->bitmaps + 3 * g->nwords;
    cudaError_t e = cudaMemsetAsync(g->bitmaps, 0, 4 * g->nwords * 4, eng->stream);
    if (e != cudaSuccess) st = fail(KITES_ERR_CUDA, "memset: %s", cudaGetErrorString(e));
  }
  if (st == KITES_OK && v->frontier_bits) {
    uint64_t words = (std::min<uint64_t>(v->frontier_nbits, g->nbits) + 31) / 32;
    cudaError_t e = cudaMemcpyAsync(g->frontier[0], v->frontier_bits, words * 4,
                                    cudaMemcpyDefault, eng->stream);
    if (e != cudaSuccess) st = fail(KITES_ERR_CUDA, "frontier copy: %s", cudaGetErrorString(e));
  }
  if (st == KITES_OK) st = graph_alloc(g, &p, 2 * sizeof(run_counters));
  if (st == KITES_OK) {
    g->ctr = (run_counters *)p;
    g->ctr_ext = g->ctr + 1;
    cudaMemsetAsync(g->ctr, 0, 2 * sizeof(run_counters), eng->stream);
    st = graph_alloc(g, &p, 2 * KITES_MAX_RECORDED_ITERS * 8);
  }
  if (st == KITES_OK) {
    g->rec_active = (unsigned long long *)p;
    g->rec_edges = g->rec_active + KITES_MAX_RECORDED_ITERS;
    cudaError_t e = cudaStreamSynchronize(eng->stream);
    if (e != cudaSuccess) st = fail(KITES_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
  }
  if (st != KITES_OK) {
    kites_graph_destroy(g);
    return st;
  }
  *out = g;
  return KITES_OK;
}

// ---- device-side ingestion (edge list -> CSC) -----------------------------

// keys[i] = dst << 32 | src; any endpoint >= n sets *bad.
__global__ void k_edge_keys(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                            uint64_t m, uint64_t n, uint64_t *__restrict__ keys, uint32_t *bad) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = src[i], d = dst[i];
    if (s >= n || d >= n) atomicOr(bad, 1u);
    keys[i] = (uint64_t)d << 32 | s;
  }
}

// R[d] = first sorted edge whose destination is >= d (binary search), for
// d in [0, n]; C[i] = source of sorted edge i.
__global__ void k_rows_of_keys(const uint64_t *__restrict__ keys, uint64_t m, uint64_t n,
                               uint64_t *__restrict__ R, uint32_t *__restrict__ C) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t d = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; d <= n; d += stride) {
    uint64_t lo = 0, hi = m;  // first index with key >> 32 >= d
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if ((keys[mid] >> 32) < d) lo = mid + 1; else hi = mid;
    }
    R[d] = lo;
  }
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
    C[i] = (uint32_t)keys[i];
}

// Builds the CSC of an edge list on the device -- rows keyed by
// destination, each row's sources ascending, parallel edges kept in input
// order (a stable radix sort of dst << 32 | src) -- and uploads it as
// kites_graph_upload does.  The edge arrays may be host or device memory.
extern "C" int kites_graph_from_edges(kites_engine *eng, uint64_t n_vertices, uint64_t n_edges,
                                      const uint32_t *src, const uint32_t *dst,
                                      const uint32_t *weights, int directed,
                                      kites_graph **out) {
  clear_error();
  if (!eng || !out) return fail(KITES_ERR_INVALID, "null argument");
  *out = nullptr;
  if (n_vertices == 0 || n_vertices >= 0xFFFFFF00ull)
    return fail(KITES_ERR_INVALID, "n_vertices must be in 1 .. 2^32 - 256");
  if (n_edges && (!src || !dst)) return fail(KITES_ERR_INVALID, "null edge arrays");
  if (n_edges > 0xFFFFFFFFull)
    return fail(KITES_ERR_UNSUPPORTED, "device ingestion takes < 2^32 edges");
  KITES_TRY(set_device(eng));
  cudaStream_t s = eng->stream;
  const uint64_t m = n_edges, n = n_vertices;
  void *p = nullptr;
  uint64_t *keys[2] = {nullptr, nullptr}, *R = nullptr;
  uint32_t *ends[2] = {nullptr, nullptr}, *w[2] = {nullptr, nullptr}, *C = nullptr, *bad = nullptr;
  void *temp = nullptr;
  std::vector<void *> tmp;
  auto alloc = [&](void **q, size_t bytes) {
    int st = dev_alloc(eng, q, bytes);
    if (st == KITES_OK) tmp.push_back(*q);
    return st;
  };
  int st = KITES_OK;
  do {
    const size_t mm = (size_t)std::max<uint64_t>(m, 1);
    if ((st = alloc(&p, mm * 8)) != KITES_OK) break;
    keys[0] = (uint64_t *)p;
    if ((st = alloc(&p, mm * 8)) != KITES_OK) break;
    keys[1] = (uint64_t *)p;
    if ((st = alloc(&p, (n + 1) * 8)) != KITES_OK) break;
    R = (uint64_t *)p;
    if ((st = alloc(&p, mm * 4)) != KITES_OK) break;
    C = (uint32_t *)p;
    if ((st = alloc(&p, 4)) != KITES_OK) break;
    bad = (uint32_t *)p;
    if (weights) {
      if ((st = alloc(&p, mm * 4)) != KITES_OK) break;
      w[0] = (uint32_t *)p;
      if ((st = alloc(&p, mm * 4)) != KITES_OK) break;
      w[1] = (uint32_t *)p;
    }
    cudaError_t e = cudaMemsetAsync(bad, 0, 4, s);
    if (m) {
      // The endpoints pass through the second key buffer (2 x 4 bytes an edge).
      ends[0] = (uint32_t *)keys[1];
      ends[1] = ends[0] + m;
      if (e == cudaSuccess) e = cudaMemcpyAsync(ends[0], src, m * 4, cudaMemcpyDefault, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(ends[1], dst, m * 4, cudaMemcpyDefault, s);
      if (e == cudaSuccess && weights)
        e = cudaMemcpyAsync(w[0], weights, m * 4, cudaMemcpyDefault, s);
      if (e != cudaSuccess) { st = fail(KITES_ERR_CUDA, "edge copy: %s", cudaGetErrorString(e)); break; }
      k_edge_keys<<<grid_for(m), 256, 0, s>>>(ends[0], ends[1], m, n, keys[0], bad);
      uint32_t hbad = 0;
      e = cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) { st = fail(KITES_ERR_CUDA, "edge keys: %s", cudaGetErrorString(e)); break; }
      if (hbad) { st = fail(KITES_ERR_INVALID, "edge endpoint >= n_vertices"); break; }
      int end_bit = 33;
      while (end_bit < 64 && (1ull << (end_bit - 32)) < n) ++end_bit;
      size_t temp_bytes = 0;
      if (weights)
        e = cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys[0], keys[1], w[0], w[1],
                                            (uint64_t)m, 0, end_bit, s);
      else
        e = cub::DeviceRadixSort::SortKeys(nullptr, temp_bytes, keys[0], keys[1], (uint64_t)m, 0,
                                           end_bit, s);
      if (e != cudaSuccess) { st = fail(KITES_ERR_CUDA, "sort: %s", cudaGetErrorString(e)); break; }
      if ((st = alloc(&temp, temp_bytes)) != KITES_OK) break;
      if (weights)
        e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys[0], keys[1], w[0], w[1],
                                            (uint64_t)m, 0, end_bit, s);
      else
        e = cub::DeviceRadixSort::SortKeys(temp, temp_bytes, keys[0], keys[1], (uint64_t)m, 0,
                                           end_bit, s);
      if (e != cudaSuccess) { st = fail(KITES_ERR_CUDA, "sort: %s", cudaGetErrorString(e)); break; }
    }
    k_rows_of_keys<<<grid_for(n + 1), 256, 0, s>>>(keys[1], m, n, R, C);
    e = cudaGetLastError();
    if (e != cudaSuccess) { st = fail(KITES_ERR_CUDA, "rows: %s", cudaGetErrorString(e)); break; }
    // The keys (16 bytes an edge), the unsorted weights and the sort's
    // scratch go back to the pool before the upload builds the graph's own
    // arrays: at 2^31 edges that is about 50 GB less at the peak.
    for (void *q : {(void *)keys[0], (void *)keys[1], (void *)w[0], temp}) {
      if (!q) continue;
      cudaFreeAsync(q, s);
      tmp.erase(std::remove(tmp.begin(), tmp.end(), q), tmp.end());
    }
    kites_csc_view v = {};
    v.n_vertices = n;
    v.n_edges = m;
    v.row_offsets = R;
    v.col_indices = C;
    v.edge_values = weights ? w[1] : nullptr;
    v.edge_value_size = weights ? 4 : 0;
    v.vertex_value_size = 4;
    v.vertex_per_group = 1;
    v.directed = directed ? 1 : 0;
    v.on_device = 1;
    st = kites_graph_upload(eng, &v, out);
  } while (0);
  for (void *q : tmp) cudaFreeAsync(q, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (st == KITES_OK && e != cudaSuccess)
    st = fail(KITES_ERR_CUDA, "ingestion: %s", cudaGetErrorString(e));
  return st;
}

extern "C" int kites_graph_device_view(kites_graph *g, kites_device_view *o) {
  clear_error();
  if (!g || !o) return fail(KITES_ERR_INVALID, "null argument");
  o->n_vertices = g->n;
  o->n_edges = g->m;
  o->nbits = g->nbits;
  o->vertex_per_group = g->vpg;
  o->directed = g->directed;
  o->offsets64 = g->off64 ? 1 : 0;
  o->V = g->V;
  o->R = g->R;
  o->C = g->C;
  o->E = g->E;
  o->dir_R = g->dirR;
  o->dir_C = g->dirC;
  o->frontier[0] = g->frontier[0];
  o->frontier[1] = g->frontier[1];
  o->update_flag = &g->ctr->update_flag;
  o->stream = (void *)g->eng->stream;
  o->changed[0] = g->changed[0];
  o->changed[1] = g->changed[1];
  o->chunk_rows = g->chunk_in;
  o->n_chunks = g->nchunks_in;
  o->chunk_items = g->chunk_items;
  return KITES_OK;
}

extern "C" int kites_graph_activate(kites_graph *g, const uint32_t *changed, uint32_t *frontier) {
  clear_error();
  if (!g || !changed || !frontier) return fail(KITES_ERR_INVALID, "null argument");
  KITES_TRY(set_device(g->eng));
  cudaStream_t s = g->eng->stream;
  if (g->off64) {
    chunk_geom<uint64_t> ga{(const uint64_t *)g->dirR, g->dirC, g->chunk_dir, g->nchunks_dir,
                            g->n_dir_rows, g->n_dir_rows + g->n_dir_edges, g->chunk_items};
    expand_args<uint64_t> ea{ga, changed, frontier, g->ctr_ext, 0u, 0u, 0ull};
    k_expand_chunked<uint64_t><<<g->expand_grid, kBlock, 0, s>>>(ea);
  } else {
    chunk_geom<uint32_t> ga{(const uint32_t *)g->dirR, g->dirC, g->chunk_dir, g->nchunks_dir,
                            g->n_dir_rows, g->n_dir_rows + g->n_dir_edges, g->chunk_items};
    expand_args<uint32_t> ea{ga, changed, frontier, g->ctr_ext, 0u, 0u, 0ull};
    k_expand_chunked<uint32_t><<<g->expand_grid, kBlock, 0, s>>>(ea);
  }
  KITES_CUDA_TRY(cudaGetLastError());
  return KITES_OK;
}

extern "C" int kites_graph_get_values(kites_graph *g, void *dst, uint64_t n) {
  clear_error();
  if (!g || !dst) return fail(KITES_ERR_INVALID, "null argument");
  if (n > g->n) return fail(KITES_ERR_INVALID, "asked for %llu values, graph has %llu",
                            (unsigned long long)n, (unsigned long long)g->n);
  KITES_TRY(set_device(g->eng));
  KITES_CUDA_TRY(cudaMemcpyAsync(dst, g->V, n * g->vsize, cudaMemcpyDefault, g->eng->stream));
  KITES_CUDA_TRY(cudaStreamSynchronize(g->eng->stream));
  return KITES_OK;
}

extern "C" int kites_graph_set_values(kites_graph *g, const void *src, uint64_t n) {
  clear_error();
  if (!g || !src) return fail(KITES_ERR_INVALID, "null argument");
  if (n > g->n) return fail(KITES_ERR_INVALID, "too many values");
  KITES_TRY(set_device(g->eng));
  KITES_CUDA_TRY(cudaMemcpyAsync(g->V, src, n * g->vsize, cudaMemcpyDefault, g->eng->stream));
  KITES_CUDA_TRY(cudaStreamSynchronize(g->eng->stream));
  return KITES_OK;
}

extern "C" int kites_graph_set_frontier(kites_graph *g, const uint32_t *bits, uint64_t nbits) {
  clear_error();
  if (!g) return fail(KITES_ERR_INVALID, "null graph");
  KITES_TRY(set_device(g->eng));
  cudaStream_t s = g->eng->stream;
  KITES_CUDA_TRY(cudaMemsetAsync(g->bitmaps, 0, 4 * g->nwords * 4, s));
  if (bits && nbits) {
    uint64_t words = (std::min<uint64_t>(nbits, g->nbits) + 31) / 32;
    KITES_CUDA_TRY(cudaMemcpyAsync(g->frontier[0], bits, words * 4, cudaMemcpyDefault, s));
  }
  KITES_CUDA_TRY(cudaStreamSynchronize(s));
  return KITES_OK;
}

extern "C" int kites_process(kites_engine *eng, kites_graph *g, int op,
                             const kites_run_opts *opts, kites_run_stats *stats) {
  clear_error();
  KITES_TRY(check_graph(eng, g));
  if (op < 0 || op > OP_PR) return fail(KITES_ERR_INVALID, "unknown operator %d", op);
  if (op == OP_PR) return fail(KITES_ERR_UNSUPPORTED, "use kites_pagerank");
  if (g->vsize != 4) return fail(KITES_ERR_UNSUPPORTED, "built-in operators need 4-byte vertex values");
  if ((op == OP_SSSP || op == OP_SSSP_WRAP) && g->esize != 4)
    return fail(KITES_ERR_UNSUPPORTED, "SSSP needs 4-byte edge values");
  kites_run_opts o = resolve_opts(opts);
  if (stats) memset(stats, 0, sizeof(*stats));
  if (o.strategy != KITES_STRATEGY_PLAIN)
    return fail(KITES_ERR_UNSUPPORTED, "strategy %d not available for kites_process", o.strategy);
  return g->off64 ? dispatch_process<uint64_t>(g, op, o, stats)
                  : dispatch_process<uint32_t>(g, op, o, stats);
}

// Runs `op` with a strategy other than PLAIN from the changed set already in
// changed[0] (graph values already initialised).
static int run_strategies(kites_engine *eng, kites_graph *g, int op, const kites_run_opts *opts,
                          kites_run_stats *stats) {
  kites_run_opts o = resolve_opts(opts);
  if (stats) memset(stats, 0, sizeof(*stats));
  if (g->vsize != 4) return fail(KITES_ERR_UNSUPPORTED, "built-in operators need 4-byte values");
  if ((op == OP_SSSP || op == OP_SSSP_WRAP) && g->esize != 4)
    return fail(KITES_ERR_UNSUPPORTED, "SSSP needs 4-byte edge values");
  if (o.strategy < KITES_STRATEGY_PLAIN || o.strategy >= KITES_STRATEGY_COUNT)
    return fail(KITES_ERR_INVALID, "unknown strategy %d", o.strategy);
  if (o.strategy == KITES_STRATEGY_MIP && !g->mip)
    return fail(KITES_ERR_INVALID,
                "KITES_STRATEGY_MIP needs the graph's block map (kites_graph_build_mipmap)");
  if (o.strategy == KITES_STRATEGY_AUTO)
    return g->off64 ? dispatch_auto<uint64_t>(g, op, o, stats)
                    : dispatch_auto<uint32_t>(g, op, o, stats);
  return g->off64 ? dispatch_flex<uint64_t>(g, op, o, stats)
                  : dispatch_flex<uint32_t>(g, op, o, stats);
}

extern "C" int kites_sssp(kites_engine *eng, kites_graph *g, int op, uint32_t source,
                          uint32_t *dist_out, const kites_run_opts *opts,
                          kites_run_stats *stats) {
  clear_error();
  KITES_TRY(check_graph(eng, g));
  if (op != OP_SSSP && op != OP_SSSP_WRAP && op != OP_BFS)
    return fail(KITES_ERR_INVALID, "kites_sssp takes SSSP, SSSP_WRAP or BFS");
  if (source >= g->n_given) return fail(KITES_ERR_INVALID, "source %u out of range", source);
  if (!g->outR) return fail(KITES_ERR_UNSUPPORTED, "graph has no out-CSR");
  cudaStream_t s = eng->stream;
  auto t0 = std::chrono::steady_clock::now();
  k_fill_u32<<<grid_for(g->n), 256, 0, s>>>((uint32_t *)g->V, g->n, kInf);
  KITES_CUDA_TRY(cudaMemsetAsync(g->bitmaps, 0, 4 * g->nwords * 4, s));
  if (opts && opts->strategy != KITES_STRATEGY_PLAIN) {
    // Strategy loop: the changed set starts as {source}.
    k_seed_changed<<<1, 32, 0, s>>>((uint32_t *)g->V, source, g->changed[0]);
    KITES_CUDA_TRY(cudaGetLastError());
    int st = run_strategies(eng, g, op, opts, stats);
    if (st != KITES_OK) return st;
    if (dist_out) {
      KITES_CUDA_TRY(cudaMemcpyAsync(dist_out, g->V, g->n_given * 4, cudaMemcpyDefault, s));
      KITES_CUDA_TRY(cudaStreamSynchronize(s));
    }
    if (stats)
      stats->host_ms = std::chrono::duration<double, std::milli>(
                           std::chrono::steady_clock::now() - t0).count();
    return KITES_OK;
  }
  if (g->off64)
    k_seed_source<uint64_t><<<32, 256, 0, s>>>((uint32_t *)g->V, (const uint64_t *)g->outR,
                                               g->outC, source, g->shift, g->frontier[0]);
  else
    k_seed_source<uint32_t><<<32, 256, 0, s>>>((uint32_t *)g->V, (const uint32_t *)g->outR,
                                               g->outC, source, g->shift, g->frontier[0]);
  KITES_CUDA_TRY(cudaGetLastError());
  int st = kites_process(eng, g, op, opts, stats);
  if (st != KITES_OK) return st;
  if (dist_out) {
    KITES_CUDA_TRY(cudaMemcpyAsync(dist_out, g->V, g->n_given * 4, cudaMemcpyDefault, s));
    KITES_CUDA_TRY(cudaStreamSynchronize(s));
  }
  if (stats) {
    stats->kernel_launches += 2;
    stats->host_ms = std::chrono::duration<double, std::milli>(
                         std::chrono::steady_clock::now() - t0).count();
  }
  return KITES_OK;
}

extern "C" int kites_cc(kites_engine *eng, kites_graph *g, uint32_t *labels_out,
                        const kites_run_opts *opts, kites_run_stats *stats) {
  clear_error();
  KITES_TRY(check_graph(eng, g));
  cudaStream_t s = eng->stream;
  auto t0 = std::chrono::steady_clock::now();
  k_iota_u32<<<grid_for(g->n), 256, 0, s>>>((uint32_t *)g->V, g->n);
  KITES_CUDA_TRY(cudaMemsetAsync(g->bitmaps, 0, 4 * g->nwords * 4, s));
  const bool strategies = opts && opts->strategy != KITES_STRATEGY_PLAIN;
  // Every vertex starts active; with a strategy loop every vertex starts
  // changed (its out-neighbours form the first frontier).
  k_all_active<<<grid_for(g->nwords), 256, 0, s>>>(strategies ? g->changed[0] : g->frontier[0],
                                                   strategies ? g->n_given : g->nbits, g->nwords);
  KITES_CUDA_TRY(cudaGetLastError());
  int st = strategies ? run_strategies(eng, g, OP_CC, opts, stats)
                      : kites_process(eng, g, OP_CC, opts, stats);
  if (st != KITES_OK) return st;
  if (labels_out) {
    KITES_CUDA_TRY(cudaMemcpyAsync(labels_out, g->V, g->n_given * 4, cudaMemcpyDefault, s));
    KITES_CUDA_TRY(cudaStreamSynchronize(s));
  }
  if (stats) {
    stats->kernel_launches += 2;
    stats->host_ms = std::chrono::duration<double, std::milli>(
                         std::chrono::steady_clock::now() - t0).count();
  }
  return KITES_OK;
}

extern "C" int kites_pagerank(kites_engine *eng, kites_graph *g, uint64_t n_real,
                              float *rank_out, const kites_run_opts *opts,
                              kites_run_stats *stats) {
  clear_error();
  KITES_TRY(check_graph(eng, g));
  if (n_real == 0 || n_real > g->n) return fail(KITES_ERR_INVALID, "bad n_real");
  kites_run_opts o = resolve_opts(opts);
  if (stats) memset(stats, 0, sizeof(*stats));
  return g->off64 ? run_pagerank<uint64_t>(g, n_real, rank_out, o, stats)
                  : run_pagerank<uint32_t>(g, n_real, rank_out, o, stats);
}

static int sssp_batch(kites_engine *eng, kites_graph *g, int op, const uint32_t *sources,
                      uint32_t k, uint32_t *dist_out, const kites_run_opts *opts,
                      kites_run_stats *stats);

extern "C" int kites_sssp_batch(kites_engine *eng, kites_graph *g, int op,
                                const uint32_t *sources, uint32_t k, uint32_t *dist_out,
                                const kites_run_opts *opts, kites_run_stats *stats) {
  clear_error();
  KITES_TRY(check_graph(eng, g));
  g->async_out = false;
  return sssp_batch(eng, g, op, sources, k, dist_out, opts, stats);
}

extern "C" int kites_sssp_batch_async(kites_engine *eng, kites_graph *g, int op,
                                      const uint32_t *sources, uint32_t k, uint32_t *dist_out,
                                      const kites_run_opts *opts, kites_run_stats *stats) {
  clear_error();
  KITES_TRY(check_graph(eng, g));
  g->async_out = true;
  const int st = sssp_batch(eng, g, op, sources, k, dist_out, opts, stats);
  g->async_out = false;
  return st;
}

static int sssp_batch(kites_engine *eng, kites_graph *g, int op, const uint32_t *sources,
                      uint32_t k, uint32_t *dist_out, const kites_run_opts *opts,
                      kites_run_stats *stats) {
  if (!sources) return fail(KITES_ERR_INVALID, "null sources");
  if (g->esize != 4 && op != OP_BFS) return fail(KITES_ERR_UNSUPPORTED, "SSSP needs 4-byte edge values");
  if (k != 16 && k != 32 && k != 64 && k != 128 && k != 256)
    return fail(KITES_ERR_INVALID, "batch size %u is not 16, 32, 64, 128 or 256", k);
  // Sources are read on the host to reject out-of-range ids before any
  // kernel indexes with them.
  uint32_t host_src[256];
  KITES_CUDA_TRY(cudaMemcpy(host_src, sources, k * 4, cudaMemcpyDefault));
  for (uint32_t i = 0; i < k; ++i)
    if (host_src[i] >= g->n_given)
      return fail(KITES_ERR_INVALID, "source %u (slot %u) out of range", host_src[i], i);
  kites_run_opts o = resolve_opts(opts, true);
  if (stats) memset(stats, 0, sizeof(*stats));
  if (o.strategy != KITES_STRATEGY_PLAIN) {
    if (o.strategy != KITES_STRATEGY_AUTO && o.strategy != KITES_STRATEGY_PUSH &&
        o.strategy != KITES_STRATEGY_PULL_ALL && o.strategy != KITES_STRATEGY_PULL_CHANGED)
      return fail(KITES_ERR_UNSUPPORTED, "strategy %d is not a batched strategy", o.strategy);
    if (!g->outE) return fail(KITES_ERR_UNSUPPORTED, "graph has no weighted out-CSR");
    return g->off64 ? dispatch_batch_flex<uint64_t>(g, op, host_src, k, dist_out, o, stats)
                    : dispatch_batch_flex<uint32_t>(g, op, host_src, k, dist_out, o, stats);
  }
  return g->off64 ? dispatch_batch<uint64_t>(g, op, host_src, k, dist_out, o, stats)
                  : dispatch_batch<uint32_t>(g, op, host_src, k, dist_out, o, stats);
}

// ---- multi-seed (multi-graph batches) --------------------------------------------

extern "C" int kites_sssp_multi_seed(kites_engine *eng, kites_graph *g, int op,
                                     const uint32_t *seeds, uint64_t n_seeds,
                                     uint32_t *dist_out, const kites_run_opts *opts,
                                     kites_run_stats *stats) {
  clear_error();
  KITES_TRY(check_graph(eng, g));
  if (op != OP_SSSP && op != OP_SSSP_WRAP && op != OP_BFS)
    return fail(KITES_ERR_INVALID, "multi-seed runs take SSSP, SSSP_WRAP or BFS");
  if (!seeds || n_seeds == 0) return fail(KITES_ERR_INVALID, "no seeds");
  std::vector<uint32_t> hs(n_seeds);
  KITES_CUDA_TRY(cudaMemcpy(hs.data(), seeds, n_seeds * 4, cudaMemcpyDefault));
  for (uint64_t i = 0; i < n_seeds; ++i)
    if (hs[i] >= g->n_given) return fail(KITES_ERR_INVALID, "seed %u out of range", hs[i]);
  cudaStream_t s = eng->stream;
  auto t0 = std::chrono::steady_clock::now();
  void *p;
  KITES_TRY(dev_alloc(eng, &p, n_seeds * 4));
  uint32_t *dseeds = (uint32_t *)p;
  KITES_CUDA_TRY(cudaMemcpyAsync(dseeds, hs.data(), n_seeds * 4, cudaMemcpyHostToDevice, s));
  k_fill_u32<<<grid_for(g->n), 256, 0, s>>>((uint32_t *)g->V, g->n, kInf);
  KITES_CUDA_TRY(cudaMemsetAsync(g->bitmaps, 0, 4 * g->nwords * 4, s));
  const bool strategies = opts && opts->strategy != KITES_STRATEGY_PLAIN;
  const unsigned blocks = (unsigned)std::min<uint64_t>(n_seeds, 65535);
  if (g->off64)
    k_seed_many<uint64_t><<<blocks, 128, 0, s>>>((uint32_t *)g->V, dseeds, n_seeds,
                                                 (const uint64_t *)g->outR, g->outC, g->shift,
                                                 strategies ? g->changed[0] : g->frontier[0],
                                                 strategies ? 1 : 0);
  else
    k_seed_many<uint32_t><<<blocks, 128, 0, s>>>((uint32_t *)g->V, dseeds, n_seeds,
                                                 (const uint32_t *)g->outR, g->outC, g->shift,
                                                 strategies ? g->changed[0] : g->frontier[0],
                                                 strategies ? 1 : 0);
  KITES_CUDA_TRY(cudaGetLastError());
  KITES_CUDA_TRY(cudaFreeAsync(dseeds, s));
  int st = strategies ? run_strategies(eng, g, op, opts, stats)
                      : kites_process(eng, g, op, opts, stats);
  if (st != KITES_OK) return st;
  if (dist_out) {
    KITES_CUDA_TRY(cudaMemcpyAsync(dist_out, g->V, g->n_given * 4, cudaMemcpyDefault, s));
    KITES_CUDA_TRY(cudaStreamSynchronize(s));
  }
  if (stats)
    stats->host_ms = std::chrono::duration<double, std::milli>(
                         std::chrono::steady_clock::now() - t0).count();
  return KITES_OK;
}

// ---- learned selector ------------------------------------------------------------

extern "C" int kites_selector_record(kites_engine *eng, kites_graph *g, int op, uint32_t source,
                                     float *features, float *times_ms, uint32_t capacity,
                                     uint32_t *n_records) {
  clear_error();
  KITES_TRY(check_graph(eng, g));
  if (!features || !times_ms || !n_records || capacity == 0)
    return fail(KITES_ERR_INVALID, "null output or zero capacity");
  if (op != OP_SSSP && op != OP_BFS && op != OP_CC)
    return fail(KITES_ERR_INVALID, "recording takes SSSP, BFS or CC");
  if (op == OP_SSSP && g->esize != 4) return fail(KITES_ERR_UNSUPPORTED, "SSSP needs 4-byte edges");
  if (op != OP_CC && source >= g->n_given) return fail(KITES_ERR_INVALID, "source out of range");
  cudaStream_t s = eng->stream;
  KITES_CUDA_TRY(cudaMemsetAsync(g->bitmaps, 0, 4 * g->nwords * 4, s));
  if (op == OP_CC) {
    k_iota_u32<<<grid_for(g->n), 256, 0, s>>>((uint32_t *)g->V, g->n);
    k_all_active<<<grid_for(g->nwords), 256, 0, s>>>(g->changed[0], g->n_given, g->nwords);
  } else {
    k_fill_u32<<<grid_for(g->n), 256, 0, s>>>((uint32_t *)g->V, g->n, kInf);
    k_seed_changed<<<1, 32, 0, s>>>((uint32_t *)g->V, source, g->changed[0]);
  }
  KITES_CUDA_TRY(cudaGetLastError());
  return g->off64 ? dispatch_record<uint64_t>(g, op, features, times_ms, capacity, n_records)
                  : dispatch_record<uint32_t>(g, op, features, times_ms, capacity, n_records);
}

static int fit_selector(kites_engine *eng, const float *features, const float *times_ms,
                        uint32_t n, uint32_t epochs, float lr, uint64_t seed, float *params_out,
                        float *final_loss, bool load);

extern "C" int kites_selector_train(kites_engine *eng, const float *features,
                                    const float *times_ms, uint32_t n, uint32_t epochs,
                                    float lr, uint64_t seed, float *params_out,
                                    float *final_loss) {
  return fit_selector(eng, features, times_ms, n, epochs, lr, seed, params_out, final_loss, true);
}

extern "C" int kites_selector_fit(kites_engine *eng, const float *features,
                                  const float *times_ms, uint32_t n, uint32_t epochs, float lr,
                                  uint64_t seed, float *params_out, float *final_loss) {
  if (!params_out) return fail(KITES_ERR_INVALID, "null params_out");
  return fit_selector(eng, features, times_ms, n, epochs, lr, seed, params_out, final_loss, false);
}

static int fit_selector(kites_engine *eng, const float *features, const float *times_ms,
                        uint32_t n, uint32_t epochs, float lr, uint64_t seed, float *params_out,
                        float *final_loss, bool load) {
  clear_error();
  if (!eng || !features || !times_ms || n == 0) return fail(KITES_ERR_INVALID, "bad arguments");
  KITES_TRY(set_device(eng));
  cudaStream_t s = eng->stream;
  // Targets: log of each class's time over PLAIN's (host arithmetic).
  std::vector<float> Y((size_t)n * kClasses);
  for (uint32_t i = 0; i < n; ++i) {
    const float t0 = std::max(times_ms[(size_t)i * kClasses], 1e-4f);
    for (int c = 0; c < kClasses; ++c)
      Y[(size_t)i * kClasses + c] = logf(std::max(times_ms[(size_t)i * kClasses + c], 1e-4f) / t0);
  }
  void *p;
  const size_t xb = (size_t)n * kFeat * 4, yb = (size_t)n * kClasses * 4;
  KITES_TRY(dev_alloc(eng, &p, xb + yb + 4 * kParams * 4 + 4));
  float *dX = (float *)p, *dY = dX + (size_t)n * kFeat, *P = dY + (size_t)n * kClasses;
  float *G = P + kParams, *M = G + kParams, *Vv = M + kParams, *loss = Vv + kParams;
  KITES_CUDA_TRY(cudaMemcpyAsync(dX, features, xb, cudaMemcpyDefault, s));
  KITES_CUDA_TRY(cudaMemcpyAsync(dY, Y.data(), yb, cudaMemcpyHostToDevice, s));
  KITES_CUDA_TRY(cudaMemsetAsync(G, 0, 3 * kParams * 4 + 4, s));
  k_mlp_init<<<8, 256, 0, s>>>(P, seed);
  k_mlp_standardise<<<1, 32, 0, s>>>(dX, n, P);
  const unsigned blocks = (n + 127) / 128;
  for (uint32_t e = 1; e <= epochs; ++e) {
    if (e == epochs) KITES_CUDA_TRY(cudaMemsetAsync(loss, 0, 4, s));
    k_mlp_grad<<<blocks, 128, 0, s>>>(dX, dY, n, P, G, loss);
    k_mlp_adam<<<(kParams + 255) / 256, 256, 0, s>>>(P, G, M, Vv, lr, 0.9f, 0.999f, 1e-8f, (int)e);
  }
  KITES_CUDA_TRY(cudaGetLastError());
  if (load)
    KITES_CUDA_TRY(cudaMemcpyAsync(eng->sel_params, P, kParams * 4, cudaMemcpyDeviceToDevice, s));
  float hloss = 0.f;
  KITES_CUDA_TRY(cudaMemcpyAsync(&hloss, loss, 4, cudaMemcpyDeviceToHost, s));
  if (params_out) KITES_CUDA_TRY(cudaMemcpyAsync(params_out, P, kParams * 4, cudaMemcpyDefault, s));
  KITES_CUDA_TRY(cudaFreeAsync(p, s));
  KITES_CUDA_TRY(cudaStreamSynchronize(s));
  if (final_loss) *final_loss = hloss;
  return KITES_OK;
}

extern "C" int kites_selector_record_batch(kites_engine *eng, kites_graph *g, int op,
                                           const uint32_t *sources, uint32_t k, float *features,
                                           float *times_ms, uint32_t capacity,
                                           uint32_t *n_records) {
  clear_error();
  KITES_TRY(check_graph(eng, g));
  if (!sources || !features || !times_ms || !n_records || capacity == 0)
    return fail(KITES_ERR_INVALID, "null argument or zero capacity");
  if (op != OP_SSSP && op != OP_BFS) return fail(KITES_ERR_INVALID, "recording takes SSSP or BFS");
  if (op == OP_SSSP && g->esize != 4) return fail(KITES_ERR_UNSUPPORTED, "SSSP needs 4-byte edges");
  if (k != 16 && k != 32 && k != 64 && k != 128 && k != 256)
    return fail(KITES_ERR_INVALID, "batch size %u is not 16, 32, 64, 128 or 256", k);
  uint32_t hs[256];
  KITES_CUDA_TRY(cudaMemcpy(hs, sources, k * 4, cudaMemcpyDefault));
  for (uint32_t i = 0; i < k; ++i)
    if (hs[i] >= g->n_given) return fail(KITES_ERR_INVALID, "source %u out of range", hs[i]);
  if (op == OP_SSSP)
    return g->off64 ? dispatch_record_batch_k<OP_SSSP, uint64_t>(g, hs, k, features, times_ms,
                                                                 capacity, n_records)
                    : dispatch_record_batch_k<OP_SSSP, uint32_t>(g, hs, k, features, times_ms,
                                                                 capacity, n_records);
  return g->off64 ? dispatch_record_batch_k<OP_BFS, uint64_t>(g, hs, k, features, times_ms,
                                                              capacity, n_records)
                  : dispatch_record_batch_k<OP_BFS, uint32_t>(g, hs, k, features, times_ms,
                                                              capacity, n_records);
}

extern "C" int kites_selector_load_batch(kites_engine *eng, const float *params,
                                         uint32_t n_params) {
  clear_error();
  if (!eng || !params) return fail(KITES_ERR_INVALID, "null argument");
  if (n_params != (uint32_t)kParams)
    return fail(KITES_ERR_INVALID, "selector has %d parameters, got %u", kParams, n_params);
  KITES_TRY(set_device(eng));
  KITES_CUDA_TRY(cudaMemcpyAsync(eng->sel_params_batch, params, kParams * 4, cudaMemcpyDefault,
                                 eng->stream));
  KITES_CUDA_TRY(cudaStreamSynchronize(eng->stream));
  return KITES_OK;
}

extern "C" int kites_selector_save_batch(kites_engine *eng, float *params, uint32_t n_params) {
  clear_error();
  if (!eng || !params) return fail(KITES_ERR_INVALID, "null argument");
  if (n_params != (uint32_t)kParams)
    return fail(KITES_ERR_INVALID, "selector has %d parameters, got %u", kParams, n_params);
  KITES_TRY(set_device(eng));
  KITES_CUDA_TRY(cudaMemcpyAsync(params, eng->sel_params_batch, kParams * 4, cudaMemcpyDefault,
                                 eng->stream));
  KITES_CUDA_TRY(cudaStreamSynchronize(eng->stream));
  return KITES_OK;
}

extern "C" int kites_selector_load(kites_engine *eng, const float *params, uint32_t n_params) {
  clear_error();
  if (!eng || !params) return fail(KITES_ERR_INVALID, "null argument");
  if (n_params != (uint32_t)kParams)
    return fail(KITES_ERR_INVALID, "selector has %d parameters, got %u", kParams, n_params);
  KITES_TRY(set_device(eng));
  KITES_CUDA_TRY(cudaMemcpyAsync(eng->sel_params, params, kParams * 4, cudaMemcpyDefault,
                                 eng->stream));
  KITES_CUDA_TRY(cudaStreamSynchronize(eng->stream));
  return KITES_OK;
}

extern "C" int kites_selector_save(kites_engine *eng, float *params, uint32_t n_params) {
  clear_error();
  if (!eng || !params) return fail(KITES_ERR_INVALID, "null argument");
  if (n_params != (uint32_t)kParams)
    return fail(KITES_ERR_INVALID, "selector has %d parameters, got %u", kParams, n_params);
  KITES_TRY(set_device(eng));
  KITES_CUDA_TRY(cudaMemcpyAsync(params, eng->sel_params, kParams * 4, cudaMemcpyDefault,
                                 eng->stream));
  KITES_CUDA_TRY(cudaStreamSynchronize(eng->stream));
  return KITES_OK;
}

extern "C" int kites_graph_set_tpv(kites_graph *g, int strategy) {
  clear_error();
  if (!g) return fail(KITES_ERR_INVALID, "null graph");
  if (strategy != KITES_STRATEGY_TPV1 && strategy != KITES_STRATEGY_TPV4 &&
      strategy != KITES_STRATEGY_TPV8 && strategy != KITES_STRATEGY_TPV32)
    return fail(KITES_ERR_INVALID, "not a threads-per-vertex strategy: %d", strategy);
  if (g->tpv_strategy != strategy) {
    // Cached AUTO loops captured the old width.
    for (auto it = g->loops.begin(); it != g->loops.end();) {
      if (it->first.strategy == 200) {
        cudaGraphExecDestroy(it->second.second);
        cudaGraphDestroy(it->second.first);
        it = g->loops.erase(it);
      } else {
        ++it;
      }
    }
    g->tpv_strategy = strategy;
  }
  return KITES_OK;
}

// ---- autotuner ------------------------------------------------------------------

namespace {

void drop_all_loops(kites_graph *g) {
  for (auto &kv : g->loops) {
    cudaGraphExecDestroy(kv.second.second);
    cudaGraphDestroy(kv.second.first);
  }
  g->loops.clear();
}

}  // namespace

extern "C" int kites_autotune(kites_engine *eng, kites_graph *g, int op, const uint32_t *sources,
                              uint32_t n_sources, uint32_t batch, kites_tune_result *out) {
  clear_error();
  KITES_TRY(check_graph(eng, g));
  if (!sources || n_sources == 0 || !out) return fail(KITES_ERR_INVALID, "bad arguments");
  if (op != OP_SSSP && op != OP_BFS) return fail(KITES_ERR_INVALID, "tuning takes SSSP or BFS");
  memset(out, 0, sizeof(*out));
  std::vector<uint32_t> src(n_sources);
  KITES_CUDA_TRY(cudaMemcpy(src.data(), sources, n_sources * 4, cudaMemcpyDefault));
  kites_run_opts o;
  kites_default_run_opts(&o);
  kites_run_stats st;
  // Runs each source once (the first run of a shape also warms its loop).
  auto time_single = [&](int strategy, float *ms) -> int {
    o.strategy = strategy;
    float total = 0.f;
    for (uint32_t i = 0; i < std::min<uint32_t>(n_sources, 4); ++i) {
      KITES_TRY(kites_sssp(eng, g, op, src[i], nullptr, &o, &st));
      KITES_TRY(kites_sssp(eng, g, op, src[i], nullptr, &o, &st));
      total += (float)st.device_ms;
    }
    *ms = total;
    ++out->trials;
    return KITES_OK;
  };
  // 1. Density thresholds of the plain loop (vpg == 1 graphs have sweeps).
  if (g->rowid) {
    const unsigned long long e_cands[] = {g->m / 64, g->m / 32, g->m / 16, g->m / 8, g->m / 4};
    const unsigned long long r_cands[] = {g->n / 128, g->n / 64, g->n / 32, g->n / 16, g->n / 8};
    float best = 1e30f;
    unsigned long long be = g->dense_edges, br = g->dense_rows;
    for (unsigned long long e : e_cands) {
      for (unsigned long long r : r_cands) {
        g->dense_edges = e;
        g->dense_rows = r;
        drop_all_loops(g);
        float ms;
        KITES_TRY(time_single(KITES_STRATEGY_PLAIN, &ms));
        if (ms < best) { best = ms; be = e; br = r; }
      }
    }
    g->dense_edges = be;
    g->dense_rows = br;
    out->plain_ms = best;
  }
  drop_all_loops(g);
  out->dense_edges = g->dense_edges;
  out->dense_rows = g->dense_rows;
  // 2. Threads per vertex of the selector's TPV class.
  if (g->vpg == 1 && g->directed) {
    const int cands[] = {KITES_STRATEGY_TPV1, KITES_STRATEGY_TPV4, KITES_STRATEGY_TPV8,
                         KITES_STRATEGY_TPV32};
    float best = 1e30f;
    int bt = g->tpv_strategy;
    for (int c : cands) {
      float ms;
      KITES_TRY(time_single(c, &ms));
      if (ms < best) { best = ms; bt = c; }
    }
    KITES_TRY(kites_graph_set_tpv(g, bt));
    out->tpv_ms = best;
  }
  out->tpv_strategy = g->tpv_strategy;
  // 3. The selector's coarse class: PULL_ALL or, on a graph with a block
  // map, the mipmapped frontier, timed as whole AUTO runs; MIP must win by
  // 2 % to replace PULL_ALL.
  if (g->mip && g->vpg == 1 && g->directed) {
    float t_all = 0.f, t_mip = 0.f;
    KITES_TRY(kites_graph_set_coarse(g, KITES_STRATEGY_PULL_ALL));
    KITES_TRY(time_single(KITES_STRATEGY_AUTO, &t_all));
    KITES_TRY(kites_graph_set_coarse(g, KITES_STRATEGY_MIP));
    KITES_TRY(time_single(KITES_STRATEGY_AUTO, &t_mip));
    const bool mip = t_mip < 0.98f * t_all;
    KITES_TRY(kites_graph_set_coarse(g, mip ? KITES_STRATEGY_MIP : KITES_STRATEGY_PULL_ALL));
    out->coarse_ms = mip ? t_mip : t_all;
  }
  out->coarse_strategy = g->coarse_strategy;
  // 4. Chunk size of the batched kernel.
  if (batch == 16 || batch == 32 || batch == 64 || batch == 128 || batch == 256) {
    std::vector<uint32_t> bs(batch);
    for (uint32_t i = 0; i < batch; ++i) bs[i] = src[i % n_sources];
    const uint32_t cands[] = {128, 256, 512, 1024, 2048};
    float best = 1e30f;
    uint32_t bc = g->batch_chunk_items ? g->batch_chunk_items : 256;
    kites_run_opts bo;
    kites_default_run_opts(&bo);
    for (uint32_t c : cands) {
      g->batch_items_req = c;  // the next batched run rebuilds its chunk table
      float total = 0.f;
      for (int rep = 0; rep < 2; ++rep) {
        KITES_TRY(kites_sssp_batch(eng, g, op, bs.data(), batch, nullptr, &bo, &st));
        if (rep) total += (float)st.device_ms;
      }
      ++out->trials;
      if (total < best) { best = total; bc = c; }
    }
    g->batch_items_req = bc;
    out->batch_ms = best;
  }
  out->batch_chunk_items = g->batch_items_req ? g->batch_items_req : 256u;
  return KITES_OK;
}

extern "C" int kites_graph_set_batch_gather(kites_graph *g, int mode) {
  clear_error();
  if (!g) return fail(KITES_ERR_INVALID, "null graph");
  if (mode < 0 || mode > 2) return fail(KITES_ERR_INVALID, "batch gather mode is 0, 1 or 2");
  KITES_TRY(set_device(g->eng));
  KITES_CUDA_TRY(cudaStreamSynchronize(g->eng->stream));
  g->batch_gather = mode;
  drop_batch_loops(g);  // captured loops hold the kernel choice
  return KITES_OK;
}

// ---- block map (mipmapped frontier) ------------------------------------------

extern "C" int kites_graph_build_mipmap(kites_graph *g, uint64_t block_vertices) {
  clear_error();
  if (!g) return fail(KITES_ERR_INVALID, "null graph");
  if (g->vpg != 1 || !g->directed)
    return fail(KITES_ERR_UNSUPPORTED,
                "the block map needs a directed graph with vertex_per_group 1");
  if (block_vertices == 0) return fail(KITES_ERR_INVALID, "block_vertices must be >= 1");
  if (g->n_given == 0) return fail(KITES_ERR_INVALID, "empty graph");
  // graph_csr_mipmapped.hpp:58-60: ceil(n / block), then up to a multiple of
  // 32, n the vertex count padded to a multiple of 128 as graph_raw pads it
  // (graph_raw.h:174-179) and as the engine holds it.
  uint64_t dim = (g->n + block_vertices - 1) / block_vertices;
  dim = (dim + 31) / 32 * 32;
  if (dim > kMaxMipDim)
    return fail(KITES_ERR_INVALID,
                "block map of %llu x %llu bits is over the %llu x %llu limit; take larger blocks",
                (unsigned long long)dim, (unsigned long long)dim,
                (unsigned long long)kMaxMipDim, (unsigned long long)kMaxMipDim);
  KITES_TRY(set_device(g->eng));
  cudaStream_t s = g->eng->stream;
  KITES_CUDA_TRY(cudaStreamSynchronize(s));
  drop_all_loops(g);   // captured loops hold the old map
  graph_release(g, g->mip);
  graph_release(g, g->mip_blocks);
  g->mip = g->mip_blocks = nullptr;
  g->mip_dim = g->mip_block = 0;
  if (g->coarse_strategy == KITES_STRATEGY_MIP) g->coarse_strategy = KITES_STRATEGY_PULL_ALL;
  const uint64_t words = dim * dim / 32;
  void *p = nullptr, *q = nullptr;
  KITES_TRY(graph_alloc(g, &p, words * 4));
  KITES_TRY(graph_alloc(g, &q, dim / 32 * 2 * 4));
  KITES_CUDA_TRY(cudaMemsetAsync(p, 0, words * 4, s));
  KITES_CUDA_TRY(cudaMemsetAsync(q, 0, dim / 32 * 2 * 4, s));
  const mip_geom mg{(uint32_t *)p, dim, dim / 32, block_vertices};
  const unsigned grid = grid_for(g->n * 32, 256, g->eng->sm_count * 16);
  if (g->off64)
    k_mip_build<uint64_t><<<grid, 256, 0, s>>>((const uint64_t *)g->R, g->C, g->n, mg);
  else
    k_mip_build<uint32_t><<<grid, 256, 0, s>>>((const uint32_t *)g->R, g->C, g->n, mg);
  KITES_CUDA_TRY(cudaGetLastError());
  KITES_CUDA_TRY(cudaStreamSynchronize(s));
  g->mip = (uint32_t *)p;
  g->mip_blocks = (uint32_t *)q;
  g->mip_dim = dim;
  g->mip_block = block_vertices;
  return KITES_OK;
}

extern "C" int kites_graph_get_mipmap(kites_graph *g, uint64_t *dim_out, uint32_t *words,
                                      uint64_t n_words) {
  clear_error();
  if (!g) return fail(KITES_ERR_INVALID, "null graph");
  if (!g->mip) return fail(KITES_ERR_INVALID, "the graph has no block map");
  if (dim_out) *dim_out = g->mip_dim;
  if (!words) return KITES_OK;
  const uint64_t total = g->mip_dim * g->mip_dim / 32;
  if (n_words < total)
    return fail(KITES_ERR_INVALID, "the block map has %llu words, the buffer %llu",
                (unsigned long long)total, (unsigned long long)n_words);
  KITES_TRY(set_device(g->eng));
  KITES_CUDA_TRY(cudaMemcpyAsync(words, g->mip, total * 4, cudaMemcpyDefault, g->eng->stream));
  KITES_CUDA_TRY(cudaStreamSynchronize(g->eng->stream));
  return KITES_OK;
}

extern "C" int kites_graph_set_coarse(kites_graph *g, int strategy) {
  clear_error();
  if (!g) return fail(KITES_ERR_INVALID, "null graph");
  if (strategy != KITES_STRATEGY_PULL_ALL && strategy != KITES_STRATEGY_MIP)
    return fail(KITES_ERR_INVALID, "the coarse class is PULL_ALL or MIP, not %d", strategy);
  if (strategy == KITES_STRATEGY_MIP && !g->mip)
    return fail(KITES_ERR_INVALID, "MIP needs the graph's block map (kites_graph_build_mipmap)");
  if (g->coarse_strategy != strategy) {
    KITES_TRY(set_device(g->eng));
    KITES_CUDA_TRY(cudaStreamSynchronize(g->eng->stream));
    drop_all_loops(g);   // cached AUTO loops captured the old class
    g->coarse_strategy = strategy;
  }
  return KITES_OK;
}

extern "C" int kites_graph_set_density(kites_graph *g, uint64_t dense_edges,
                                       uint64_t dense_rows) {
  clear_error();
  if (!g) return fail(KITES_ERR_INVALID, "null graph");
  KITES_TRY(set_device(g->eng));
  KITES_CUDA_TRY(cudaStreamSynchronize(g->eng->stream));
  g->dense_edges = dense_edges;
  g->dense_rows = dense_rows;
  drop_all_loops(g);  // captured loops hold the old thresholds
  return KITES_OK;
}
