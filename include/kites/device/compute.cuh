// compute.cuh -- kites::process, the iterate-to-fixed-point driver of the
// kites:: API (farkhor/KiTES kites/device/compute.cuh:29-137, 397-411).
//
// With user lambdas the iteration kernel is instantiated here, in the
// caller's translation unit (generic_kernels.cuh), and driven by the same
// host loop as the reference: clear the device flag, launch, clear the read
// frontier, read the flag back, repeat while it is set.  With a built-in
// operator tag (kites::ops::*) the call goes to the engine's precompiled
// edge-balanced kernels and device-side loop (kites_process).
#ifndef KITES_B200_COMPUTE_CUH_
#define KITES_B200_COMPUTE_CUH_

#include <chrono>
#include <iostream>

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
  cudaStream_t s = (cudaStream_t)dv.stream;
  const uint64_t nwords = (dv.nbits + 31) / 32;
  const unsigned grid = (unsigned)(dv.n_vertices / (generic::kWarps * 32));
  uint32_t shift = 0;
  while ((1u << shift) < dv.vertex_per_group) ++shift;
  // Activation adjacency: the out-adjacency, or C itself for undirected graphs.
  const void *actR = dv.directed ? dv.dir_R : dv.R;
  const uint32_t *actC = dv.directed ? dv.dir_C : dv.C;
  std::cout << "Launching iterative procedure ...\n";
  auto t0 = std::chrono::steady_clock::now();
  unsigned iterations = 0;
  unsigned *hflag = g.updateFlagHost.get_ptr();
  do {
    CUDAErrorCheck(cudaMemsetAsync(dv.update_flag, 0, sizeof(unsigned), s));
    const bool even = (iterations & 1) == 0;
    uint32_t *rd = dv.frontier[even ? 0 : 1];
    uint32_t *wr = dv.frontier[even ? 1 : 0];
    if (dv.offsets64)
      generic::pull_iteration<vT, eT, uint64_t><<<grid, generic::kWarps * 32, 0, s>>>(
          dv.n_vertices, (const uint64_t *)dv.R, dv.C, (vT *)dv.V, (eT *)dv.E, dv.update_flag,
          rd, wr, shift, (const uint64_t *)actR, actC, fInit, fComp, fRed, fUpd);
    else
      generic::pull_iteration<vT, eT, uint32_t><<<grid, generic::kWarps * 32, 0, s>>>(
          dv.n_vertices, (const uint32_t *)dv.R, dv.C, (vT *)dv.V, (eT *)dv.E, dv.update_flag,
          rd, wr, shift, (const uint32_t *)actR, actC, fInit, fComp, fRed, fUpd);
    CUDAErrorCheck(cudaPeekAtLastError());
    generic::clear_words<<<(unsigned)((nwords + 255) / 256), 256, 0, s>>>(rd, nwords);
    CUDAErrorCheck(cudaMemcpyAsync(hflag, dv.update_flag, sizeof(unsigned),
                                   cudaMemcpyDeviceToHost, s));
    ++iterations;
    CUDAErrorCheck(cudaStreamSynchronize(s));
  } while (*hflag != 0);
  const double ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  std::cout << "Processing finished in " << ms << " (ms).\n";
  std::cout << "Performed " << iterations << " iterations in total.\n";
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
