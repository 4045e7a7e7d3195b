// compute.cuh -- kites::process, the iterate-to-fixed-point driver of the
// kites:: API (farkhor/KiTES kites/device/compute.cuh:29-137, 397-411).
//
// With user lambdas the iteration kernels are instantiated here, in the
// caller's translation unit (generic_kernels.cuh), over the engine's
// edge-balanced chunk table, and the whole loop runs on the device: one CUDA
// graph whose conditional while node repeats {pull, join the split rows,
// activation (the engine's kites_graph_activate), clear, check} until no
// vertex changed -- the reference's host round trip per iteration
// (compute.cuh:57-128) becomes a device-side test.  With a built-in operator
// tag (kites::ops::*) the call goes to the engine's precompiled kernels
// (kites_process).
#ifndef KITES_B200_COMPUTE_CUH_
#define KITES_B200_COMPUTE_CUH_

#include <chrono>
#include <iostream>
#include <stdexcept>
#include <string>

#include "../../kites_b200.h"
#include "../common/globals.cuh"
#include "../graph/graph_csr_device.cuh"
#include "../graph/graph_csr_mipmapped_device.cuh"
#include "generic_kernels.cuh"
#include "nv_gpu.cuh"

namespace kites {

// Built-in operators (the engine's precompiled vertex programs).
namespace ops {
struct builtin_op { int op; };
constexpr builtin_op sssp{KITES_OP_SSSP};            // saturating min-plus
constexpr builtin_op sssp_wrap{KITES_OP_SSSP_WRAP};  // the example's wrap-around add
constexpr builtin_op bfs{KITES_OP_BFS};
constexpr builtin_op cc{KITES_OP_CC};
}  // namespace ops

namespace detail {

// Enqueues one iteration of the user program on stream s (parity p reads
// frontier p, writes frontier p ^ 1) and the loop check.
template <class vT, class eT, class OffT, class FInit, class FComp, class FRed, class FUpd>
void enqueue_generic_iteration(kites_graph *h, const kites_device_view &dv, int p,
                               generic::chunk_args<vT, OffT> a, unsigned grid,
                               cudaGraphConditionalHandle cond, generic::loop_state *ls,
                               FInit &fInit, FComp &fComp, FRed &fRed, FUpd &fUpd,
                               cudaStream_t s) {
  a.rd = dv.frontier[p];
  a.chg = dv.changed[p];
  const uint64_t nwords = (dv.nbits + 31) / 32;
  generic::chunk_pull<vT, eT, OffT><<<grid, generic::kWarps * 32, 0, s>>>(
      a, (vT *)dv.V, (eT *)dv.E, fInit, fComp, fRed, fUpd);
  generic::combine_split_rows<vT, eT, OffT><<<(unsigned)((a.n_chunks + 127) / 128), 128, 0, s>>>(
      a, (vT *)dv.V, fInit, fRed, fUpd);
  KITESErrorCheck(kites_graph_activate(h, dv.changed[p], dv.frontier[p ^ 1]));
  generic::clear_two<<<(unsigned)((nwords + 255) / 256), 256, 0, s>>>(dv.frontier[p],
                                                                       dv.changed[p], nwords);
  generic::loop_check<<<1, 1, 0, s>>>(dv.update_flag, ls, cond);
}

}  // namespace detail

template <launch launchMode, class vT, class eT, class vIdxT, class FInit, class FComp,
          class FRed, class FUpd>
void process(graph_csr_device<vT, eT, vIdxT> &g, nv_gpu &dev, FInit fInit, FComp fComp,
             FRed fRed, FUpd fUpd) {
  dev.setAsActive();
  const auto mem = dev.queryMemUsage();
  std::cout << mem.first << " MB is consumed out of the total " << mem.second
            << " MB global memory.\n";
  kites_device_view dv{};
  KITESErrorCheck(kites_graph_device_view(g.engine_graph(), &dv));
  if (dv.offsets64) throw std::runtime_error("kites::process takes 32-bit row offsets");
  cudaStream_t s = (cudaStream_t)dv.stream;
  uint32_t shift = 0;
  while ((1u << shift) < dv.vertex_per_group) ++shift;
  const uint64_t nwords = (dv.nbits + 31) / 32;

  // Per-call scratch: two fold slots per chunk and the loop state.
  vT *part = nullptr;
  uint8_t *part_has = nullptr;
  generic::loop_state *ls = nullptr;
  CUDAErrorCheck(cudaMallocAsync((void **)&part, 2 * dv.n_chunks * sizeof(vT), s));
  CUDAErrorCheck(cudaMallocAsync((void **)&part_has, 2 * dv.n_chunks, s));
  CUDAErrorCheck(cudaMallocAsync((void **)&ls, sizeof(generic::loop_state), s));
  generic::loop_state init{};
  // A monotone program settles within n + 1 rounds; the cap only ends one
  // that cannot converge.
  init.max_iterations = 2 * dv.n_vertices + 16;
  CUDAErrorCheck(cudaMemcpyAsync(ls, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  CUDAErrorCheck(cudaMemsetAsync(dv.update_flag, 0, sizeof(uint32_t), s));
  CUDAErrorCheck(cudaMemsetAsync(dv.changed[0], 0, nwords * 4, s));
  CUDAErrorCheck(cudaMemsetAsync(dv.changed[1], 0, nwords * 4, s));

  generic::chunk_args<vT, uint32_t> a{};
  a.R = (const uint32_t *)dv.R;
  a.C = dv.C;
  a.chunk_rows = dv.chunk_rows;
  a.n_chunks = dv.n_chunks;
  a.n_rows = dv.n_vertices;
  a.chunk_items = dv.chunk_items;
  a.shift = shift;
  a.flag = dv.update_flag;
  a.part = part;
  a.part_has = part_has;
  a.ls = ls;
  int per_sm = 0, sms = 0, devi = 0;
  CUDAErrorCheck(cudaGetDevice(&devi));
  CUDAErrorCheck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, devi));
  CUDAErrorCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, generic::chunk_pull<vT, eT, uint32_t, FInit, FComp, FRed, FUpd>,
      generic::kWarps * 32, 0));
  const uint64_t want = (dv.n_chunks + generic::kWarps - 1) / generic::kWarps;
  const uint64_t cap = (uint64_t)(per_sm > 0 ? per_sm : 1) * (uint64_t)sms;
  const unsigned grid = (unsigned)(want < cap ? (want ? want : 1) : cap);

  // while (not converged) { iteration(even); iteration(odd) }
  cudaGraph_t graph;
  CUDAErrorCheck(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle cond;
  CUDAErrorCheck(cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  CUDAErrorCheck(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
  CUDAErrorCheck(cudaStreamBeginCaptureToGraph(s, cp.conditional.phGraph_out[0], nullptr,
                                               nullptr, 0, cudaStreamCaptureModeRelaxed));
  for (int p = 0; p < 2; ++p)
    detail::enqueue_generic_iteration<vT, eT, uint32_t>(g.engine_graph(), dv, p, a, grid, cond,
                                                        ls, fInit, fComp, fRed, fUpd, s);
  cudaGraph_t captured;
  CUDAErrorCheck(cudaStreamEndCapture(s, &captured));
  cudaGraphExec_t exec;
  CUDAErrorCheck(cudaGraphInstantiate(&exec, graph, 0));

  std::cout << "Launching iterative procedure ...\n";
  cudaEvent_t e0, e1;
  CUDAErrorCheck(cudaEventCreate(&e0));
  CUDAErrorCheck(cudaEventCreate(&e1));
  auto t0 = std::chrono::steady_clock::now();
  CUDAErrorCheck(cudaEventRecord(e0, s));
  CUDAErrorCheck(cudaGraphLaunch(exec, s));
  CUDAErrorCheck(cudaEventRecord(e1, s));
  generic::loop_state fin{};
  CUDAErrorCheck(cudaMemcpyAsync(&fin, ls, sizeof(fin), cudaMemcpyDeviceToHost, s));
  CUDAErrorCheck(cudaStreamSynchronize(s));
  const double ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  float dms = 0.f;
  CUDAErrorCheck(cudaEventElapsedTime(&dms, e0, e1));
  g.last_device_ms = dms;
  g.last_iterations = fin.iterations;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  CUDAErrorCheck(cudaFreeAsync(part, s));
  CUDAErrorCheck(cudaFreeAsync(part_has, s));
  CUDAErrorCheck(cudaFreeAsync(ls, s));
  CUDAErrorCheck(cudaStreamSynchronize(s));
  if (fin.timed_out)
    throw std::runtime_error("kites::process: no fixed point after " +
                             std::to_string(fin.iterations) + " iterations");
  std::cout << "Processing finished in " << ms << " (ms).\n";
  std::cout << "Performed " << fin.iterations << " iterations in total.\n";
}

// Mipmapped graphs: coarse activation (the reference declares the mipmapped
// graph classes, kites/graph/graph_csr_mipmapped*.{hpp,cuh}, but no process
// overload consumes them).  The frontier holds one bit per block of
// compressionRatio vertices; every vertex of an active block pulls with the
// user functions, and a block with an updated vertex activates every block
// its mipmap row names.  That activates a superset of the vertices the
// per-vertex out-adjacency would, so a monotone program (min-plus,
// min-label, BFS levels) reaches the same fixed point as over graph_csr.
// Same host loop as above: clear the flag, launch, clear the read frontier,
// read the flag back.
template <launch launchMode, class vT, class eT, class vIdxT, class FInit, class FComp,
          class FRed, class FUpd>
void process(graph_csr_mipmapped_device<vT, eT, vIdxT> &g, nv_gpu &dev, FInit fInit,
             FComp fComp, FRed fRed, FUpd fUpd) {
  dev.setAsActive();
  const auto mem = dev.queryMemUsage();
  std::cout << mem.first << " MB is consumed out of the total " << mem.second
            << " MB global memory.\n";
  cudaStream_t s = dev.getSsEven().get();
  const uint64_t n = g.get_num_vertices();
  const uint32_t words = g.mipmapDim / 32;
  const unsigned grid = (unsigned)(n / (generic::kWarps * 32));
  const dim3 egrid((words + 127) / 128,
                   (g.mipmapDim + generic::kMipRowsPerSlice - 1) / generic::kMipRowsPerSlice);
  std::cout << "Launching iterative procedure ...\n";
  auto t0 = std::chrono::steady_clock::now();
  unsigned iterations = 0;
  unsigned *hflag = g.updateFlagHost.get_ptr();
  do {
    CUDAErrorCheck(cudaMemsetAsync(g.updateFlag.get_ptr(), 0, sizeof(unsigned), s));
    CUDAErrorCheck(cudaMemsetAsync(g.changedBlocks.get_ptr(), 0, words * sizeof(unsigned), s));
    const bool even = (iterations & 1) == 0;
    uint32_t *rd = even ? g.vBitmapEven.get_ptr() : g.vBitmapOdd.get_ptr();
    uint32_t *wr = even ? g.vBitmapOdd.get_ptr() : g.vBitmapEven.get_ptr();
    if (grid)
      generic::mip_pull_iteration<vT, eT><<<grid, generic::kWarps * 32, 0, s>>>(
          n, g.R.get_ptr(), g.C.get_ptr(), g.V.get_ptr(), g.E.get_ptr(), g.updateFlag.get_ptr(),
          rd, g.compressionRatio, g.changedBlocks.get_ptr(), fInit, fComp, fRed, fUpd);
    CUDAErrorCheck(cudaPeekAtLastError());
    if (words) {
      generic::mip_expand<<<egrid, 128, 0, s>>>(g.mipmap.get_ptr(), words,
                                                g.changedBlocks.get_ptr(), wr);
      CUDAErrorCheck(cudaPeekAtLastError());
      generic::clear_words<<<(words + 255) / 256, 256, 0, s>>>(rd, words);
    }
    CUDAErrorCheck(cudaMemcpyAsync(hflag, g.updateFlag.get_ptr(), sizeof(unsigned),
                                   cudaMemcpyDeviceToHost, s));
    ++iterations;
    CUDAErrorCheck(cudaStreamSynchronize(s));
  } while (*hflag != 0);
  const double ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  std::cout << "Processing finished in " << ms << " (ms).\n";
  std::cout << "Performed " << iterations << " iterations in total.\n";
}

// Built-in operator: the engine's precompiled kernels and device-side loop.
template <launch launchMode, class vT, class eT, class vIdxT>
kites_run_stats process(graph_csr_device<vT, eT, vIdxT> &g, nv_gpu &dev, ops::builtin_op op,
                        const kites_run_opts *opts = nullptr) {
  dev.setAsActive();
  kites_run_stats st{};
  KITESErrorCheck(kites_process(dev.engine(), g.engine_graph(), op.op, opts, &st));
  return st;
}

// Host-graph convenience overload (compute.cuh:397-411): upload, process,
// copy V back into the host graph.
template <launch launchMode, class vT, class eT, class vIdxT, class FInit, class FComp,
          class FRed, class FUpd>
void process(graph_csr<vT, eT, vIdxT> &h, nv_gpu &dev, FInit fInit, FComp fComp, FRed fRed,
             FUpd fUpd) {
  auto d = make_graph_csr_for_device(h, dev);
  process<launch::sync>(d, dev, fInit, fComp, fRed, fUpd);
  copyMem(h.V, d.V);
}

}  // namespace kites

#endif
