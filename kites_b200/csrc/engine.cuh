// engine.cuh -- engine and device-graph objects behind the C ABI.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <map>
#include <utility>
#include <vector>

#include "common.cuh"

struct kites_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t kev0 = nullptr, kev1 = nullptr;   // per-kernel timing
  // Asynchronous batch results: device-to-host copies run on copy_stream
  // (staged = the staging buffer holds a result, copied = its copy is done).
  cudaStream_t copy_stream = nullptr;
  cudaStream_t copy_stream2 = nullptr;  // the second half of each copy
  cudaEvent_t staged = nullptr, copied = nullptr, copied2 = nullptr;
  cudaMemPool_t pool = nullptr;   // stream-ordered pool owning every buffer
  int sm_count = 0;
  int l2_bytes = 0;
  void *pinned = nullptr;         // small pinned scratch for flag read-backs
  float *sel_params = nullptr;    // learned selector weights (device), or null
  float *sel_params_batch = nullptr;  // the batched loop's selector weights
  std::vector<struct kites_graph *> graphs;   // live graphs, destroyed with the engine
};

namespace kites_internal {

struct loop_key {
  int op;
  int strategy;
  bool operator<(const loop_key &o) const {
    return op != o.op ? op < o.op : strategy < o.strategy;
  }
};

}  // namespace kites_internal

struct kites_graph {
  kites_engine *eng = nullptr;
  uint64_t n = 0;          // padded vertex count (multiple of 128)
  uint64_t n_given = 0;    // rows in the uploaded CSC
  uint64_t m = 0;
  uint32_t vpg = 1, shift = 0;
  int directed = 1;
  bool off64 = false;      // row arrays are uint64
  uint32_t vsize = 4, esize = 4;

  void *R = nullptr;       // OffT[n+1]
  uint32_t *C = nullptr;   // [m]
  void *E = nullptr;       // [m] x esize
  void *V = nullptr;       // [n] x vsize

  // Vertex-level out-CSR with weights (rows = sources), built on device.
  void *outR = nullptr;
  uint32_t *outC = nullptr;
  uint32_t *outE = nullptr;
  uint32_t *out_deg = nullptr;   // [n] out-degree per vertex

  // Activation adjacency (dir_R / dir_C; rows = vertices or groups).
  void *dirR = nullptr;
  uint32_t *dirC = nullptr;
  uint64_t n_dir_rows = 0, n_dir_edges = 0;

  // Edge-balanced chunk tables.
  uint32_t chunk_items = 2048;
  uint32_t *chunk_in = nullptr;
  uint64_t nchunks_in = 0;
  uint32_t *chunk_dir = nullptr;
  uint64_t nchunks_dir = 0;

  // Row of every in-edge, for the edge-parallel dense sweeps (vpg == 1 only).
  uint32_t *rowid = nullptr;
  int sweep_grid = 0;
  unsigned long long dense_edges = 0;   // PLAIN switches to the sweep above this
  unsigned long long dense_rows = 0;    // activation switches to the sweep above this

  // Frontier: [f0 | c0 | f1 | c1], nwords each.
  uint32_t *bitmaps = nullptr;
  uint64_t nbits = 0, nwords = 0;
  uint32_t *frontier[2] = {nullptr, nullptr};
  uint32_t *changed[2] = {nullptr, nullptr};

  kites_internal::run_counters *ctr = nullptr;
  kites_internal::run_counters *ctr_ext = nullptr;  // kites_graph_activate's (never done)
  unsigned long long *rec_active = nullptr;
  unsigned long long *rec_edges = nullptr;

  // Batched multi-source runs (V x K distances), allocated on first use.
  uint32_t *batchD = nullptr;
  uint64_t batch_cap = 0;            // elements of batchD
  uint32_t *stage = nullptr;         // kites_sssp_batch_async: the last result, for copy_stream
  uint64_t stage_cap = 0;
  bool async_out = false;            // the running batch call delivers through stage
  uint32_t *bbits = nullptr;         // vertex-level [f0|c0|f1|c1] when vpg > 1
  uint64_t bnwords = 0;
  uint32_t batch_chunk_items = 0;    // chunk size chunk_batch was built with
  uint32_t batch_items_req = 0;      // chunk size asked for (autotuner), 0 = 256
  uint32_t *chunk_batch = nullptr;
  uint64_t nchunks_batch = 0;
  uint32_t *chunk_out = nullptr;     // vertex-level out-CSR chunks (vpg > 1)
  uint64_t nchunks_out = 0;
  uint32_t *d_sources = nullptr;     // 256 source slots
  // TMA view of batchD (K-wide rows) for the gather kernel; batch_gather:
  // 2 = cp.async row copies into shared memory (default: R-MAT scale 24,
  // learned + batched 291.0 against 254.3 GTEPS with register loads, 305
  // with six rows in flight per lane group at four CTAs per SM),
  // 1 = TMA row gathers when K >= 32, 0 = register loads.
  CUtensorMap dmap;
  const void *dmap_ptr = nullptr;
  uint32_t dmap_K = 0;
  int batch_gather = 2;
  uint32_t *bmask = nullptr;         // batched strategies: changed sectors per vertex,
                                     // two parities of n words
  uint32_t *queue = nullptr;         // compacted changed queue (PUSH), n slots
  void *sacc = nullptr;              // selector frontier-count accumulators
  uint8_t *rec_sel = nullptr;        // selector class per iteration (device)
  int tpv_strategy = KITES_STRATEGY_TPV8;   // the selector's threads-per-vertex class
  int coarse_strategy = KITES_STRATEGY_PULL_ALL;  // the selector's coarse class (or MIP)
  // Block map of the mipmapped frontier (KITES_STRATEGY_MIP): mip_dim x
  // mip_dim bits, row = source block; mip_blocks holds the changed-block and
  // active-block bitmaps (mip_dim / 32 words each).
  uint32_t *mip = nullptr;
  uint32_t *mip_blocks = nullptr;
  uint64_t mip_dim = 0, mip_block = 0;
  float auto_margin = -1.f;          // margin the cached AUTO loop was captured with
  float auto_margin_batch = -1.f;    // the same for the batched AUTO loops

  // PageRank scratch (allocated on first use).
  float *pr_x = nullptr, *pr_y = nullptr, *pr_inv_out = nullptr;

  // time_kernels: one record per iteration of the last host-loop run (pull
  // time, whether the dense sweep did the pull, the counters after it).
  struct pull_rec {
    float ms;
    bool dense;
    bool fused;   // the pull also found its rows from the previous changed set
    unsigned long long active, edges, total_updated;
  };
  std::vector<pull_rec> pull_log;

  // Instantiated device loops (conditional while graphs), per op/strategy.
  std::map<kites_internal::loop_key, std::pair<cudaGraph_t, cudaGraphExec_t>> loops;

  std::vector<void *> owned;   // every pool allocation of this graph
  int pull_grid = 0, expand_grid = 0;
};
