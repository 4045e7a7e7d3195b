// engine.cu -- C ABI of the B200 vertex-centric engine: engine/graph
// lifetimes, device layout build, and the iteration loops of the built-in
// vertex programs (host-driven as in kites/device/compute.cuh:57-128, or a
// CUDA graph with a conditional while node and device-side convergence).
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "engine.cuh"
#include "kernels.cuh"
#include "kernels_pr.cuh"

using namespace kites_internal;

namespace kites_internal {

char *error_buffer() {
  static thread_local char buf[512];
  return buf;
}

namespace {

int dev_alloc(kites_engine *eng, void **p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) bytes = 256;
  bytes = (bytes + 255) & ~size_t(255);
  cudaError_t e = cudaMallocFromPoolAsync(p, bytes, eng->pool, eng->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(KITES_ERR_OOM, "device pool allocation of %zu bytes failed: %s",
                bytes, cudaGetErrorString(e));
  }
  return KITES_OK;
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
  if (m > 0x7FFFFFFFull)
    return fail(KITES_ERR_UNSUPPORTED, "out-CSR build supports < 2^31 edges");
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
                                               (OffT *)g->outR, (int)(n + 1), s));
  void *temp;
  KITES_TRY(dev_alloc(eng, &temp, temp_bytes));
  KITES_CUDA_TRY(cub::DeviceScan::ExclusiveSum(temp, temp_bytes, deg_wide,
                                               (OffT *)g->outR, (int)(n + 1), s));
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
                                                 idx_in, idx_out, (int)m, 0, end_bit, s));
  KITES_TRY(dev_alloc(eng, &temp, temp_bytes));
  KITES_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, g->C, keys_out,
                                                 idx_in, idx_out, (int)m, 0, end_bit, s));
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
  return KITES_OK;
}

// ---- iteration loops ----------------------------------------------------

struct loop_ctx {
  kites_graph *g;
  int op;
};

template <int OP, typename OffT>
int launch_iteration(kites_graph *g, int parity, cudaGraphConditionalHandle h,
                     int has_handle, uint64_t *launches, bool time_pull = false) {
  cudaStream_t s = g->eng->stream;
  if (time_pull) KITES_CUDA_TRY(cudaEventRecord(g->eng->kev0, s));
  chunk_geom<OffT> gin{(const OffT *)g->R, g->C, g->chunk_in, g->nchunks_in,
                       g->n, g->n + g->m, g->chunk_items};
  pull_args<OffT> pa{gin, (const uint32_t *)g->E, (uint32_t *)g->V,
                     g->frontier[parity], g->changed[parity], g->shift, g->ctr};
  k_pull_chunked<OP, OffT><<<g->pull_grid, kBlock, 0, s>>>(pa);
  if (time_pull) KITES_CUDA_TRY(cudaEventRecord(g->eng->kev1, s));
  chunk_geom<OffT> gdir{(const OffT *)g->dirR, g->dirC, g->chunk_dir, g->nchunks_dir,
                        g->n_dir_rows, g->n_dir_rows + g->n_dir_edges, g->chunk_items};
  expand_args<OffT> ea{gdir, g->changed[parity], g->frontier[parity ^ 1], g->ctr};
  k_expand_chunked<OffT><<<g->expand_grid, kBlock, 0, s>>>(ea);
  // Clear the read frontier and the changed bitmap (adjacent words).
  k_clear_words<<<grid_for(2 * g->nwords, 256, 4096), 256, 0, s>>>(g->frontier[parity],
                                                                    2 * g->nwords);
  iter_record rec{g->rec_active, g->rec_edges, KITES_MAX_RECORDED_ITERS};
  k_loop_check<<<1, 1, 0, s>>>(g->ctr, rec, h, has_handle);
  KITES_CUDA_TRY(cudaGetLastError());
  *launches += 4;
  return KITES_OK;
}

template <int OP, typename OffT>
int get_device_loop(kites_graph *g, int strategy, cudaGraphExec_t *exec) {
  loop_key key{OP, strategy};
  auto it = g->loops.find(key);
  if (it != g->loops.end()) {
    *exec = it->second.second;
    return KITES_OK;
  }
  cudaStream_t s = g->eng->stream;
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
  int st = launch_iteration<OP, OffT>(g, 0, handle, 1, &dummy);
  if (st == KITES_OK) st = launch_iteration<OP, OffT>(g, 1, handle, 1, &dummy);
  cudaGraph_t captured;
  cudaError_t e = cudaStreamEndCapture(s, &captured);
  if (st != KITES_OK) return st;
  KITES_CUDA_TRY(e);
  cudaGraphExec_t ex;
  KITES_CUDA_TRY(cudaGraphInstantiate(&ex, graph, 0));
  g->loops[key] = {graph, ex};
  *exec = ex;
  return KITES_OK;
}

struct pinned_state {
  uint32_t done;
  uint32_t timed_out;
  unsigned long long iterations;
};

template <int OP, typename OffT>
int run_plain(kites_graph *g, const kites_run_opts &o, kites_run_stats *st) {
  kites_engine *eng = g->eng;
  cudaStream_t s = eng->stream;
  auto t0 = std::chrono::steady_clock::now();
  run_counters init = {};
  // A monotone program reaches its fixed point within n + 1 rounds; the
  // default cap only ends a loop that cannot converge (e.g. a wrapping add
  // from 0xFFFFFFFF), with KITES_ERR_TIMEOUT.
  init.max_iterations = o.max_iterations ? o.max_iterations : 2 * g->n + 16;
  run_counters *hctr = (run_counters *)eng->pinned;
  *hctr = init;
  KITES_CUDA_TRY(cudaMemcpyAsync(g->ctr, hctr, sizeof(run_counters),
                                 cudaMemcpyHostToDevice, s));
  uint64_t launches = 0;
  KITES_CUDA_TRY(cudaEventRecord(eng->ev0, s));
  if (o.device_loop && !o.time_kernels) {
    cudaGraphExec_t ex;
    KITES_TRY((get_device_loop<OP, OffT>(g, KITES_STRATEGY_PLAIN, &ex)));
    KITES_CUDA_TRY(cudaGraphLaunch(ex, s));
  } else {
    // Host-driven loop, one flag read-back per iteration (compute.cuh:57-128).
    for (uint64_t it = 0;; ++it) {
      KITES_TRY((launch_iteration<OP, OffT>(g, (int)(it & 1), 0, 0, &launches,
                                            o.time_kernels != 0)));
      KITES_CUDA_TRY(cudaMemcpyAsync(hctr, g->ctr, sizeof(run_counters),
                                     cudaMemcpyDeviceToHost, s));
      KITES_CUDA_TRY(cudaStreamSynchronize(s));
      if (o.time_kernels && st) {
        float kms = 0.f;
        KITES_CUDA_TRY(cudaEventElapsedTime(&kms, eng->kev0, eng->kev1));
        st->pull_kernel_ms += kms;
        st->pull_kernel_launches += 1;
      }
      if (hctr->done) break;
    }
  }
  KITES_CUDA_TRY(cudaEventRecord(eng->ev1, s));
  KITES_CUDA_TRY(cudaMemcpyAsync(hctr, g->ctr, sizeof(run_counters),
                                 cudaMemcpyDeviceToHost, s));
  KITES_CUDA_TRY(cudaStreamSynchronize(s));
  float ms = 0.f;
  KITES_CUDA_TRY(cudaEventElapsedTime(&ms, eng->ev0, eng->ev1));
  const bool dev_loop = o.device_loop && !o.time_kernels;
  if (dev_loop) launches = 4 * hctr->iterations;  // kernels that ran
  if (st) {
    st->iterations = hctr->iterations;
    st->device_ms = ms;
    st->edges_traversed = hctr->total_edges;
    const uint64_t e_bytes = op_reads_weights<OP>() ? 4 : 0;
    // Algorithmic bytes (plain pull): per iteration 2 x 4 ceil(nbits/32) for
    // the bitmap read and reset, 12 B per active vertex, (4 + eT + vT) per
    // traversed in-edge, vT + 8 per updated row and 8 per activation edge.
    const uint64_t bitmap = 8ull * ((g->nbits + 31) / 32);
    st->algorithmic_bytes = hctr->iterations * bitmap + 12ull * hctr->total_active +
                            (8ull + e_bytes) * hctr->total_edges +
                            12ull * hctr->total_updated + 8ull * hctr->total_out_edges;
    st->strategy_hist[KITES_STRATEGY_PLAIN] += hctr->iterations;
    if (o.time_kernels)
      // Pull kernel alone: frontier words, 12 B per active vertex (V[v],
      // R[v], R[v+1]), (4 C + eT + 4 V[src]) per in-edge, 4 B per store.
      st->pull_kernel_bytes = hctr->iterations * 4ull * ((g->nbits + 31) / 32) +
                              12ull * hctr->total_active +
                              (8ull + e_bytes) * hctr->total_edges +
                              4ull * hctr->total_updated;
    st->kernel_launches += launches;
    if (o.record_iterations) {
      uint32_t nrec = (uint32_t)std::min<unsigned long long>(hctr->iterations,
                                                             KITES_MAX_RECORDED_ITERS);
      st->n_recorded = nrec;
      if (nrec) {
        KITES_CUDA_TRY(cudaMemcpy(st->iter_active, g->rec_active, nrec * 8,
                                  cudaMemcpyDeviceToHost));
        KITES_CUDA_TRY(cudaMemcpy(st->iter_edges, g->rec_edges, nrec * 8,
                                  cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < nrec; ++i) st->iter_strategy[i] = KITES_STRATEGY_PLAIN;
      }
    }
  }
  if (hctr->timed_out)
    return fail(KITES_ERR_TIMEOUT, "no fixed point after %llu iterations",
                (unsigned long long)hctr->iterations);
  auto t1 = std::chrono::steady_clock::now();
  if (st) st->host_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
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

int check_graph(kites_engine *eng, kites_graph *g) {
  if (!eng || !g) return fail(KITES_ERR_INVALID, "null engine or graph");
  if (g->eng != eng) return fail(KITES_ERR_INVALID, "graph belongs to another engine");
  return set_device(eng);
}

kites_run_opts resolve_opts(const kites_run_opts *opts) {
  kites_run_opts o;
  kites_default_run_opts(&o);
  if (opts) o = *opts;
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
  o->selector_margin = 0.1f;
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
        (ce = cudaEventCreate(&eng->kev1)) != cudaSuccess) {
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
  // Graphs die with their engine; their handles are invalid afterwards.
  while (!eng->graphs.empty()) kites_graph_destroy(eng->graphs.back());
  if (eng->pinned) cudaFreeHost(eng->pinned);
  if (eng->ev0) cudaEventDestroy(eng->ev0);
  if (eng->ev1) cudaEventDestroy(eng->ev1);
  if (eng->kev0) cudaEventDestroy(eng->kev0);
  if (eng->kev1) cudaEventDestroy(eng->kev1);
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
  return KITES_OK;
}

extern "C" int kites_graph_destroy(kites_graph *g) {
  if (!g) return KITES_OK;
  cudaSetDevice(g->eng->device);
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
  g->off64 = g->m > 0xFFFFFFFFull - g->n;
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
  if (st == KITES_OK) st = graph_alloc(g, &p, sizeof(run_counters));
  if (st == KITES_OK) {
    g->ctr = (run_counters *)p;
    cudaMemsetAsync(g->ctr, 0, sizeof(run_counters), eng->stream);
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
  k_all_active<<<grid_for(g->nwords), 256, 0, s>>>(g->frontier[0], g->nbits, g->nwords);
  KITES_CUDA_TRY(cudaGetLastError());
  int st = kites_process(eng, g, OP_CC, opts, stats);
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

extern "C" int kites_sssp_batch(kites_engine *eng, kites_graph *g, int op,
                                const uint32_t *sources, uint32_t k, uint32_t *dist_out,
                                const kites_run_opts *opts, kites_run_stats *stats) {
  clear_error();
  (void)eng; (void)g; (void)op; (void)sources; (void)k; (void)dist_out; (void)opts;
  (void)stats;
  return fail(KITES_ERR_UNSUPPORTED, "batched SSSP is not built yet");
}
