/*
 * kites_b200.h -- C ABI of the B200 vertex-centric engine.
 *
 * Plain pointers and sizes only; every call returns a kites_status (0 = ok)
 * and leaves a message for kites_last_error_string() on failure.  The C++
 * front-end in include/kites/ (the drop-in for farkhor/KiTES's API) calls
 * these entry points and turns a non-zero status into std::runtime_error,
 * as the reference's CUDAErrorCheck does (kites/common/cuda_error_check.cuh:9-18).
 *
 * Each declaration names the reference interface it replaces
 * (paths relative to the KiTES project root).
 */
#ifndef KITES_B200_H_
#define KITES_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KITES_B200_ABI_VERSION 3

typedef enum kites_status {
  KITES_OK = 0,
  KITES_ERR_INVALID = 1,       /* bad argument / size / vpg not a power of 2 */
  KITES_ERR_OOM = 2,           /* device or pinned allocation failed         */
  KITES_ERR_CUDA = 3,          /* a CUDA runtime call failed                  */
  KITES_ERR_TIMEOUT = 4,       /* iteration limit or bounded wait exhausted   */
  KITES_ERR_UNSUPPORTED = 5,   /* operator/strategy combination not offered   */
  KITES_ERR_NO_DEVICE = 6      /* no CUDA device / not an sm_100 part         */
} kites_status;

/* Built-in vertex programs.  Each one is a set of the reference's four user
 * functions (README.md:14-24) with a precompiled sm_100a kernel:
 *   SSSP       init copy, partial = src + w saturating at 0xFFFFFFFF, min, <
 *   SSSP_WRAP  same with u32 wrap-around add (the example's lambda verbatim,
 *              examples/sssp_basic_single_device.cu:42-43)
 *   BFS        partial = src + 1 saturating, min, <
 *   CC         partial = src (min label), min, <
 *   PAGERANK   FP32, 20 synchronous (Jacobi) iterations by default          */
typedef enum kites_op {
  KITES_OP_SSSP = 0,
  KITES_OP_SSSP_WRAP = 1,
  KITES_OP_BFS = 2,
  KITES_OP_CC = 3,
  KITES_OP_PAGERANK = 4
} kites_op;

/* Per-iteration traversal strategies.  PLAIN is the pull iteration over the
 * bitmap frontier (kites/device/kernels_single_device.cuh:18-426 re-designed);
 * AUTO lets the learned selector pick per iteration, falling back to PLAIN
 * when the predicted gain is under the margin.  The others force one
 * strategy for every iteration (used to record training timings).
 * Batched runs (kites_sssp_batch) take PLAIN, AUTO, PUSH, PULL_ALL and
 * PULL_CHANGED; there PUSH and PULL_CHANGED move only the 32-byte sectors of
 * each source row that changed in the previous iteration, and PULL_ALL
 * pulls every row without an activation pass. */
typedef enum kites_strategy {
  KITES_STRATEGY_PLAIN = 0,
  KITES_STRATEGY_AUTO = 1,
  KITES_STRATEGY_PUSH = 2,      /* push over the compacted changed queue     */
  KITES_STRATEGY_PULL_ALL = 3,  /* dense pull sweep over every vertex        */
  KITES_STRATEGY_TPV1 = 4,      /* pull, 1 thread per active vertex          */
  KITES_STRATEGY_TPV4 = 5,      /* pull, 4 threads per active vertex         */
  KITES_STRATEGY_TPV8 = 6,      /* pull, 8 threads per active vertex         */
  KITES_STRATEGY_TPV32 = 7,     /* pull, one warp per active vertex          */
  KITES_STRATEGY_PULL_CHANGED = 8,  /* pull over the frontier, reading only
                                       in-neighbours that changed last time  */
  KITES_STRATEGY_MIP = 9,       /* pull over the vertex blocks that the graph's
                                   block map activates (needs
                                   kites_graph_build_mipmap)                 */
  KITES_STRATEGY_COUNT = 10
} kites_strategy;

typedef struct kites_engine kites_engine;
typedef struct kites_graph kites_graph;

/* A host- or device-resident CSC graph as kites::graph_csr holds it
 * (kites/graph/graph_csr.h:28-39): rows are destinations, col_indices are
 * the sources of each row's in-edges sorted ascending.  Exactly one of
 * row_offsets / row_offsets32 is non-NULL; likewise for the out-adjacency.
 * If out_col_indices is NULL and vertex_per_group == 1 the engine derives
 * the out-adjacency from the CSC itself. */
typedef struct kites_csc_view {
  uint64_t n_vertices;              /* rows; engine pads to a multiple of 128 */
  uint64_t n_edges;
  const uint64_t *row_offsets;      /* R  [n_vertices + 1]                    */
  const uint32_t *row_offsets32;
  const uint32_t *col_indices;      /* C  [n_edges]                           */
  const void *edge_values;          /* E  [n_edges] x edge_value_size, or NULL */
  uint32_t edge_value_size;         /* bytes per edge value (0 if none)       */
  uint32_t vertex_value_size;       /* bytes per vertex value                 */
  const void *vertex_values;        /* V  [n_vertices] initial values or NULL */
  uint32_t vertex_per_group;        /* vpg, a power of two                    */
  int32_t directed;                 /* kites::graph_property::directed == 1   */
  const uint32_t *frontier_bits;    /* vBitmap words (LSB = lowest id) or NULL */
  uint64_t frontier_nbits;          /* bits in vBitmap                        */
  uint64_t n_out_rows;              /* dir_R entries - 1                      */
  const uint64_t *out_row_offsets;  /* dir_R                                  */
  const uint32_t *out_row_offsets32;
  const uint32_t *out_col_indices;  /* dir_C                                  */
  uint64_t n_out_edges;
  int32_t on_device;                /* 1 if every pointer above is device memory */
  int32_t offsets64;                /* 1: keep row offsets in uint64 on the device even
                                       when uint32 would do (the layout graphs past
                                       2^32 vertices + edges get) */
} kites_csc_view;

/* Device pointers of an uploaded graph, for the header-side generic kernels
 * (the C++ front-end instantiates user lambdas in the caller's TU). */
typedef struct kites_device_view {
  uint64_t n_vertices;              /* padded */
  uint64_t n_edges;
  uint64_t nbits;                   /* frontier bits (vertices or groups) */
  uint32_t vertex_per_group;
  int32_t directed;
  int32_t offsets64;                /* 1 if row arrays are uint64 */
  void *V;
  const void *R;
  const uint32_t *C;
  void *E;
  const void *dir_R;
  const uint32_t *dir_C;
  uint32_t *frontier[2];            /* even / odd bitmaps */
  uint32_t *update_flag;            /* one device word */
  void *stream;                     /* cudaStream_t the engine works on */
  uint32_t *changed[2];             /* changed-row bitmaps, the frontier's size */
  const uint32_t *chunk_rows;       /* edge-balanced chunks of the CSC: chunk k
                                       starts at item k * chunk_items of the
                                       sequence "row v, then its in-edges" and
                                       chunk_rows[k] is the row holding that
                                       item (n_chunks + 1 entries) */
  uint64_t n_chunks;
  uint32_t chunk_items;
} kites_device_view;

typedef struct kites_run_opts {
  int32_t strategy;                 /* kites_strategy */
  int32_t device_loop;              /* 1: iteration loop captured in a CUDA
                                       graph with device-side convergence;
                                       0: host loop, flag read back per trip
                                       (compute.cuh:57-128)                  */
  uint64_t max_iterations;          /* 0 = until convergence                */
  uint32_t pagerank_iterations;     /* PAGERANK only (default 20)           */
  float damping;                    /* PAGERANK only (default 0.85)         */
  float selector_margin;            /* AUTO: min predicted gain (fraction);
                                       negative (default): 0.1 single-source,
                                       0.03 batched                          */
  int32_t record_iterations;        /* fill kites_run_stats.iter_* arrays   */
  int32_t time_kernels;             /* host loop with CUDA events around each
                                       pull launch (fills pull_kernel_*)    */
} kites_run_opts;

#define KITES_MAX_RECORDED_ITERS 4096

typedef struct kites_run_stats {
  uint64_t iterations;              /* kernel iterations, as compute.cuh:135 counts */
  double device_ms;                 /* CUDA-event time of the iteration loop */
  double host_ms;                   /* wall time of the whole call           */
  uint64_t edges_traversed;         /* sum over iterations of in-edges of active vertices */
  uint64_t algorithmic_bytes;       /* sum over iterations of B_t            */
  uint64_t strategy_hist[KITES_STRATEGY_COUNT];
  uint64_t kernel_launches;         /* engine kernels launched by the call   */
  double pull_kernel_ms;            /* time_kernels: summed pull-kernel time */
  uint64_t pull_kernel_launches;
  uint64_t pull_kernel_bytes;       /* algorithmic bytes of those launches   */
  uint32_t n_recorded;
  uint8_t iter_strategy[KITES_MAX_RECORDED_ITERS];
  float iter_ms[KITES_MAX_RECORDED_ITERS];     /* time_kernels: each pull's time */
  uint64_t iter_active[KITES_MAX_RECORDED_ITERS];
  uint64_t iter_edges[KITES_MAX_RECORDED_ITERS];
  double pull_dense_ms;             /* time_kernels, PLAIN: the pulls of the
                                       iterations the dense sweep ran       */
  uint64_t pull_dense_launches;
  uint64_t pull_dense_bytes;        /* algorithmic bytes of those launches   */
} kites_run_stats;

/* ---- library / engine ------------------------------------------------ */

/* Message of the last failed call on this host thread ("" if none). */
const char *kites_last_error_string(void);
int kites_abi_version(void);
void kites_default_run_opts(kites_run_opts *opts);

/* Replaces kites::nv_gpu(int) (kites/device/nv_gpu.cuh:32-37): binds the
 * device, creates the engine's streams and its pooled allocator. */
int kites_engine_create(int device, kites_engine **out);
int kites_engine_destroy(kites_engine *eng);
/* Replaces nv_gpu::queryMemUsage (nv_gpu.cuh:78-86), in bytes. */
int kites_engine_mem_usage(kites_engine *eng, uint64_t *used, uint64_t *total,
                           uint64_t *pool_reserved);
/* nv_gpu::sync (nv_gpu.cuh:45-48): waits for the engine stream and for the
 * copies of kites_sssp_batch_async. */
int kites_engine_sync(kites_engine *eng);
/* Orders the engine stream after every copy kites_sssp_batch_async has
 * issued so far, without blocking the host (no reference counterpart). */
int kites_engine_join(kites_engine *eng);
/* The cudaStream_t every engine call is ordered on; replaces
 * nv_gpu::getSsEven (nv_gpu.cuh:56-58), the reference's working stream. */
int kites_engine_stream(kites_engine *eng, void **stream_out);

/* ---- graphs ----------------------------------------------------------- */

/* Replaces kites::make_graph_csr_for_device / graph_csr_device's constructor
 * (kites/graph/graph_csr_device.cuh:83-152): copies the CSC, the initial
 * values and the initial frontier to the device and builds the engine's
 * B200 layout (edge-balanced chunk table, weighted out-CSR). */
int kites_graph_upload(kites_engine *eng, const kites_csc_view *view,
                       kites_graph **out);
/* Builds the CSC of an edge list on the device and uploads it, like
 * kites_graph_upload of the CSC that graph_raw::construct_me
 * (kites/graph/graph_raw.h:57-190) sorts on the host: rows keyed by
 * destination, each row's sources ascending, parallel edges kept in input
 * order.  src, dst, weights (NULL: unweighted): n_edges uint32 each, host or
 * device memory; n_edges < 2^32.  directed = 0 expects both directions of
 * every undirected edge in the list; vpg 1, vertex values 4 bytes, no
 * initial values or frontier (set them with kites_graph_set_*). */
int kites_graph_from_edges(kites_engine *eng, uint64_t n_vertices, uint64_t n_edges,
                           const uint32_t *src, const uint32_t *dst, const uint32_t *weights,
                           int directed, kites_graph **out);
int kites_graph_destroy(kites_graph *g);
int kites_graph_device_view(kites_graph *g, kites_device_view *out);
/* Copy vertex values in or out (host or device pointer, cudaMemcpyDefault),
 * as host_pinned_buffer<vT>(devGrph.V) does (host_pinned_buffer.cuh:52-57). */
int kites_graph_get_values(kites_graph *g, void *dst, uint64_t n_vertices);
int kites_graph_set_values(kites_graph *g, const void *src, uint64_t n_vertices);
int kites_graph_set_frontier(kites_graph *g, const uint32_t *bits, uint64_t nbits);
/* Enqueues on the engine's stream, without waiting, the activation step of
 * the reference's iteration (kites/device/kernels_single_device.cuh:154-167,
 * 288-324): for every row set in `changed` (vertex or group bits, device
 * memory), OR the bits of its activation-adjacency targets (dir_R/dir_C, or
 * C for undirected graphs) into `frontier`.  Allocates nothing and may be
 * captured into a CUDA graph; the C++ front-end's process() for user
 * functions calls it between its own pull kernels. */
int kites_graph_activate(kites_graph *g, const uint32_t *changed, uint32_t *frontier);

/* ---- runs --------------------------------------------------------------- */

/* kites::process<launch::sync>(devGrph, dev, initF, nbrCompF, redF, updF)
 * (kites/device/compute.cuh:29-137) for a built-in operator: iterates the
 * graph's own vertex values from its current frontier to the fixed point,
 * in place, on the device. */
int kites_process(kites_engine *eng, kites_graph *g, int op,
                  const kites_run_opts *opts, kites_run_stats *stats);

/* Single-source SSSP/BFS from `source`: sets V = INF except V[source] = 0 and
 * the frontier to source's out-neighbours (the example's pre-processing,
 * examples/sssp_basic_single_device.cu:9-27), runs kites_process, and copies
 * the distances to `dist_out` (host or device) if it is non-NULL. */
int kites_sssp(kites_engine *eng, kites_graph *g, int op, uint32_t source,
               uint32_t *dist_out, const kites_run_opts *opts,
               kites_run_stats *stats);

/* Batched multi-source SSSP/BFS: K sources at once, distances in a
 * V x K vertex-major array (dist_out[v*K + k]); K is 16, 32, 64, 128 or 256.
 * opts->strategy: PLAIN (the K-wide pull every iteration), or -- for the
 * saturating SSSP and BFS on graphs with vertex_per_group 1 -- AUTO (the
 * batched learned selector), PUSH, PULL_ALL or PULL_CHANGED. */
int kites_sssp_batch(kites_engine *eng, kites_graph *g, int op,
                     const uint32_t *sources, uint32_t k, uint32_t *dist_out,
                     const kites_run_opts *opts, kites_run_stats *stats);

/* The same, returning as soon as the distances are computed: they are
 * copied on the device into a per-graph staging buffer (n x K values, kept
 * by the graph) and from there to dist_out on a second stream, so the next
 * batch computes while this one's result crosses to the host (give pinned
 * host memory for the copy to overlap).  dist_out must not be read before
 * kites_engine_sync (or, on the device side, kites_engine_join) and must
 * stay valid until then.  No reference counterpart. */
int kites_sssp_batch_async(kites_engine *eng, kites_graph *g, int op,
                           const uint32_t *sources, uint32_t k, uint32_t *dist_out,
                           const kites_run_opts *opts, kites_run_stats *stats);

/* Multi-seed SSSP/BFS: every seed starts at 0 (one super-source).  On a
 * disjoint union of graphs with one seed per member this runs a whole batch
 * of independent graphs in one device loop (multi-graph batching); each
 * member's distances equal its own single-source result.  No reference
 * counterpart beyond process() itself. */
int kites_sssp_multi_seed(kites_engine *eng, kites_graph *g, int op, const uint32_t *seeds,
                          uint64_t n_seeds, uint32_t *dist_out, const kites_run_opts *opts,
                          kites_run_stats *stats);

/* Single-source saturating SSSP that allocates no device memory, for callers
 * that cannot allocate when they need an answer (memory reserved up front
 * with allocation forbidden on the serving path, or device memory owned by
 * another runtime's allocator).  No counterpart in the reference.
 * The caller owns every buffer: the CSC (R: n+1 uint32 offsets, C, E:
 * n_edges uint32), the out-adjacency (out_R, out_C: destinations of each
 * source, n_edges entries) and dist (n uint32), all device pointers; stream
 * may be NULL.  Scratch (two frontier bitmaps, flags) is a fixed 4 MiB + 256 B
 * array compiled into the library, held by every GPU that loads it until the
 * process exits; hence n_vertices <= 16,777,216 (larger sizes are rejected).
 * The first call on a device looks that array's address up and should come
 * before any stream capture.  Calls share the array: calls that overlap on
 * the GPU race.  Validates the graph on the device before traversing it. */
int kites_sssp_noalloc(const uint32_t *R, const uint32_t *C, const uint32_t *E, uint64_t n_edges,
                       const uint32_t *out_R, const uint32_t *out_C, uint32_t n_vertices,
                       uint32_t source, uint32_t *dist, void *stream, uint32_t *iterations);

/* Min-label connected components: V[v] = v, every vertex active. */
int kites_cc(kites_engine *eng, kites_graph *g, uint32_t *labels_out,
             const kites_run_opts *opts, kites_run_stats *stats);

/* FP32 PageRank, `opts->pagerank_iterations` Jacobi steps of
 * PR <- (1-d)/n_real + d * sum PR(u)/outdeg(u), uniform 1/n_real start. */
int kites_pagerank(kites_engine *eng, kites_graph *g, uint64_t n_real,
                   float *rank_out, const kites_run_opts *opts,
                   kites_run_stats *stats);

/* ---- learned strategy selector ---------------------------------------
 * No reference counterpart: the reference always runs its one pull kernel.
 * A 12 -> 32 -> 32 -> 4 FP32 MLP predicts, from frontier statistics, the
 * log time ratio of each strategy class (PLAIN, PUSH, PULL_ALL, TPV) to
 * PLAIN for the next iteration; KITES_STRATEGY_AUTO runs the class with the
 * lowest prediction when it beats PLAIN by more than opts->selector_margin,
 * else PLAIN.  An engine starts with neutral weights (always PLAIN). */
#define KITES_SELECTOR_FEATURES 12
#define KITES_SELECTOR_CLASSES 4
#define KITES_SELECTOR_PARAMS 1628

/* Training data: single-source run (or CC when op == KITES_OP_CC) where every
 * iteration first times each class from the same state (then restores it)
 * and then advances with PLAIN.  features: capacity x 12, times_ms:
 * capacity x 4 (PLAIN, PUSH, PULL_ALL, TPV). */
int kites_selector_record(kites_engine *eng, kites_graph *g, int op, uint32_t source,
                          float *features, float *times_ms, uint32_t capacity,
                          uint32_t *n_records);
/* Full-batch Adam on MSE of log(t_class / t_PLAIN), hand-written CUDA
 * kernels; loads the result into the engine and copies it to params_out. */
int kites_selector_train(kites_engine *eng, const float *features, const float *times_ms,
                         uint32_t n_records, uint32_t epochs, float learning_rate,
                         uint64_t seed, float *params_out, float *final_loss);
int kites_selector_load(kites_engine *eng, const float *params, uint32_t n_params);
int kites_selector_save(kites_engine *eng, float *params, uint32_t n_params);
/* The same fit, returning the parameters without loading them anywhere. */
int kites_selector_fit(kites_engine *eng, const float *features, const float *times_ms,
                       uint32_t n_records, uint32_t epochs, float learning_rate, uint64_t seed,
                       float *params_out, float *final_loss);
/* The batched loop's selector (kites_sssp_batch with KITES_STRATEGY_AUTO):
 * the same MLP and features over the batch's changed set, with its own
 * weights; classes PLAIN, PUSH, PULL_ALL, PULL_CHANGED.  Training data: a
 * K-source batched run where every iteration times each class from the
 * same state (D, changed set and changed sectors restored after each) and
 * then advances with PLAIN; times_ms: capacity x 4 in class order. */
int kites_selector_record_batch(kites_engine *eng, kites_graph *g, int op,
                                const uint32_t *sources, uint32_t k, float *features,
                                float *times_ms, uint32_t capacity, uint32_t *n_records);
int kites_selector_load_batch(kites_engine *eng, const float *params, uint32_t n_params);
int kites_selector_save_batch(kites_engine *eng, float *params, uint32_t n_params);
/* Threads-per-vertex width of the selector's TPV class for this graph
 * (KITES_STRATEGY_TPV1/4/8/32). */
int kites_graph_set_tpv(kites_graph *g, int strategy);
/* What the selector's coarse class (class 2) runs on this graph:
 * KITES_STRATEGY_PULL_ALL (default) or KITES_STRATEGY_MIP (needs the block
 * map).  The autotuner picks it on graphs with a block map. */
int kites_graph_set_coarse(kites_graph *g, int strategy);

/* ---- mipmapped frontier ------------------------------------------------
 * The block map of kites::graph_csr_mipmapped (kites/graph/
 * graph_csr_mipmapped.hpp:58-75, uploaded by graph_csr_mipmapped_device,
 * graph_csr_mipmapped_device.cuh:44-64), built on the device from the
 * uploaded CSC: blocks of block_vertices consecutive vertices, dim =
 * ceil(n / block_vertices) rounded up to a multiple of 32 (n the vertex
 * count padded to a multiple of 128, as graph_raw.h:174-179 pads it), and a
 * dim x dim row-major bit matrix with bit
 * (s / block_vertices) * dim + d / block_vertices set for every edge s -> d
 * (bit b of the matrix is bit b % 32 of word b / 32).  dim <= 65536.
 * KITES_STRATEGY_MIP activates, after each iteration, every vertex of every
 * block that a block holding a changed vertex has an edge into.  Directed
 * graphs with vertex_per_group 1.  Rebuilding replaces the map. */
int kites_graph_build_mipmap(kites_graph *g, uint64_t block_vertices);
/* dim of the map, and its dim * dim / 32 words if words is non-NULL
 * (n_words: the buffer's capacity, host or device memory). */
int kites_graph_get_mipmap(kites_graph *g, uint64_t *dim_out, uint32_t *words,
                           uint64_t n_words);

/* ---- autotuner ---------------------------------------------------------
 * No reference counterpart (the reference fixes 128 threads per block and
 * one vertex per thread).  Times candidate tile shapes on this graph with
 * the given sources and keeps the fastest: the batched kernel's chunk size
 * (vertices + edges per warp), the threads-per-vertex width of the
 * selector's TPV class, its coarse class (PULL_ALL or MIP, on graphs with a
 * block map), and the frontier densities at which the plain loop
 * switches its pull and its activation to the staged sweeps. */
typedef struct kites_tune_result {
  uint32_t batch_chunk_items;
  int32_t tpv_strategy;
  uint64_t dense_edges;
  uint64_t dense_rows;
  float batch_ms;          /* best batched run time             */
  float plain_ms;          /* best plain single-source run time */
  float tpv_ms;            /* best TPV single-source run time   */
  uint32_t trials;
  int32_t coarse_strategy; /* the selector's coarse class: PULL_ALL or MIP */
  float coarse_ms;         /* its AUTO run time (graphs with a block map) */
} kites_tune_result;

int kites_autotune(kites_engine *eng, kites_graph *g, int op, const uint32_t *sources,
                   uint32_t n_sources, uint32_t batch, kites_tune_result *out);
/* Sets the two densities by hand: the plain loop's pull uses the staged sweep
 * when the activation edges exceed dense_edges, its activation when the
 * changed rows exceed dense_rows (0 = always, UINT64_MAX = never). */
int kites_graph_set_density(kites_graph *g, uint64_t dense_edges, uint64_t dense_rows);
/* How kites_sssp_batch fetches the K-wide source rows (no counterpart in the
 * reference, whose kernels run one source at a time): 2 (default) = per-lane
 * cp.async copies into shared memory (the fixed batched loop, and the pulls
 * and the push of the batched strategies), 0 = 256-bit register loads,
 * 1 = TMA tile::gather4 copies into shared memory when K >= 32 (the fixed
 * batched loop only).  All give identical results. */
int kites_graph_set_batch_gather(kites_graph *g, int mode);

/* ---- synthetic graphs (host, deterministic, OpenMP) ------------------ */

/* Candidate edges come from a counter-based SplitMix64 stream; self-loops,
 * out-of-range ids (n_vertices < 2^scale) and duplicate pairs are dropped
 * and the list is topped up from further candidates until n_edges remain.
 * Output is in candidate order.  Weights uniform in [w_lo, w_hi]. */
int kites_gen_rmat(uint32_t scale, uint64_t n_vertices, uint64_t n_edges,
                   double a, double b, double c, uint64_t seed, uint32_t w_lo,
                   uint32_t w_hi, uint32_t *src, uint32_t *dst, uint32_t *w);
int kites_gen_er(uint64_t n_vertices, uint64_t n_edges, uint64_t seed,
                 uint32_t w_lo, uint32_t w_hi, uint32_t *src, uint32_t *dst,
                 uint32_t *w);
/* side x side 4-neighbour grid, both directions, 2*2*side*(side-1) edges. */
int kites_gen_grid(uint32_t side, uint64_t seed, uint32_t w_lo, uint32_t w_hi,
                   uint32_t *src, uint32_t *dst, uint32_t *w);
/* Disjoint union of n_graphs R-MAT graphs for multi-graph batches: graph i
 * has V_i log-uniform in [v_min, v_max], edge factor uniform in
 * [ef_min, ef_max]; its vertex ids start at vertex_offsets[i] and its edges
 * at edge_offsets[i] (both n_graphs + 1 entries).  src == NULL: sizes only. */
int kites_gen_rmat_union(uint32_t n_graphs, uint64_t seed, uint32_t v_min, uint32_t v_max,
                         uint32_t ef_min, uint32_t ef_max, uint32_t w_lo, uint32_t w_hi,
                         uint64_t *vertex_offsets, uint64_t *edge_offsets, uint32_t *src,
                         uint32_t *dst, uint32_t *w);
/* Edge list -> CSC keyed by destination, rows sorted by source (ties in
 * input order), graph_raw.h:102,131 semantics; R has n_vertices+1 entries. */
int kites_csc_from_edges(uint64_t n_vertices, uint64_t n_edges,
                         const uint32_t *src, const uint32_t *dst,
                         const uint32_t *w, uint64_t *R, uint32_t *C,
                         uint32_t *E);

/* ---- binary CSC files ------------------------------------------------
 * The reference's prepared format is text, one value per line
 * (kites/io/graph_output.cuh:23-38, read back by the graph_csr(file)
 * constructor, kites/graph/graph_csr.h:112-166); these keep the same CSC
 * (R, C, E) as raw arrays behind a 128-byte header, so that a large graph is
 * built once and read back in seconds.  Layout: "KITESCSC", uint32 version 1,
 * uint32 flags (1: edge values, 2: directed), uint64 n_vertices, uint64
 * n_edges, uint64 0, char desc[88]; then R (n_vertices + 1 uint64), C and E
 * (n_edges uint32 each).  A file is written under a temporary name and
 * renamed into place. */
int kites_csc_save(const char *path, uint64_t n_vertices, uint64_t n_edges,
                   const uint64_t *R, const uint32_t *C, const uint32_t *E, int directed,
                   const char *desc);
/* Sizes and flags of a CSC file; desc (may be NULL) receives its description. */
int kites_csc_info(const char *path, uint64_t *n_vertices, uint64_t *n_edges,
                   int *has_values, int *directed, char *desc, size_t desc_len);
/* Reads a CSC file into caller arrays sized from kites_csc_info (E may be
 * NULL to skip the edge values). */
int kites_csc_load(const char *path, uint64_t *R, uint32_t *C, uint32_t *E);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* KITES_B200_H_ */
