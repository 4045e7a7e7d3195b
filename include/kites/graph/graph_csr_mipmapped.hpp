// graph_csr_mipmapped.hpp -- the host graph with a coarse activation map
// (farkhor/KiTES kites/graph/graph_csr_mipmapped.hpp:16-113).
//
// Vertices are grouped into blocks of `compressionRatio` consecutive ids.
// `mipmap` is a mipmapDim x mipmapDim bit matrix, row-major: bit
// a * mipmapDim + b is set iff a vertex of block a has an out-edge to a
// vertex of block b (graph_csr_mipmapped.hpp:74-75).  `vBitmap` is the
// initial frontier with one bit per block: block v / compressionRatio is set
// iff the pre-processing function activated vertex v (:71-72).
// mipmapDim = ceil(n / compressionRatio) rounded up to a multiple of 32,
// with n the 128-padded vertex count (:57-60).  V, R, C, E are built by the
// same rules as graph_csr's directed one-vertex-per-group constructor (the
// reference builds both through graph_raw with vpg = 1).
#ifndef KITES_B200_GRAPH_CSR_MIPMAPPED_HPP_
#define KITES_B200_GRAPH_CSR_MIPMAPPED_HPP_

#include <cmath>
#include <fstream>
#include <stdexcept>
#include <string>
#include <utility>

#include "../common/globals.cuh"
#include "../io/file_interactor.hpp"
#include "../memory/host_pinned_buffer.cuh"
#include "graph_base.h"
#include "graph_csr.h"

namespace kites {

template <class vT, class eT, class vIdxT = unsigned int>
class graph_csr_mipmapped : public graph_base {
  using eIdxT = vIdxT;

 public:
  host_pinned_buffer<vT> V;
  host_pinned_buffer<eIdxT> R;
  host_pinned_buffer<vIdxT> C;
  host_pinned_buffer<eT> E;
  host_pinned_buffer<unsigned int> updateFlag;

  unsigned int compressionRatio;
  unsigned int mipmapDim = 0;
  host_bitmap vBitmap;
  host_bitmap mipmap;

  template <class funcT>
  graph_csr_mipmapped(std::ifstream &inputFile, funcT f, unsigned int const compressionRatioIn,
                      input_graph_form const gForm = input_graph_form::edge_list_s_d)
      : compressionRatio{compressionRatioIn} {
    construct(inputFile, f, gForm);
  }
  template <class funcT>
  graph_csr_mipmapped(std::string const inputFileStr, funcT f,
                      unsigned int const compressionRatioIn,
                      input_graph_form const gForm = input_graph_form::edge_list_s_d)
      : compressionRatio{compressionRatioIn} {
    std::ifstream inputFile;
    io::openFileToAccess(inputFile, inputFileStr);
    construct(inputFile, f, gForm);
  }

 private:
  template <class funcT>
  void construct(std::ifstream &in, funcT f, input_graph_form gForm) {
    if (compressionRatio == 0) throw std::runtime_error("compression ratio must be positive");
    // The CSC, the padded V, the per-vertex frontier and the out-adjacency.
    graph_csr<vT, eT, vIdxT> g(in, f, gForm, graph_property::directed,
                               edge_list_expression::complete);
    const std::size_t n = g.get_num_vertices();
    set_num_vertices(n);
    set_num_edges(g.get_num_edges());
    V = std::move(g.V);
    R = std::move(g.R);
    C = std::move(g.C);
    E = std::move(g.E);
    updateFlag.alloc(1);
    updateFlag[0] = 0;
    const std::size_t blocks = (n + compressionRatio - 1) / compressionRatio;
    mipmapDim = static_cast<unsigned int>((blocks + 31) / 32 * 32);
    vBitmap.alloc(mipmapDim);
    vBitmap.reset();
    mipmap.alloc(static_cast<std::size_t>(mipmapDim) * mipmapDim);
    mipmap.reset();
    for (std::size_t v = 0; v < n; ++v) {
      if (g.vBitmap.getAt(v)) vBitmap.setAt(v / compressionRatio);
      const std::size_t row = (v / compressionRatio) * mipmapDim;
      for (std::size_t k = g.dir_R[v]; k < g.dir_R[v + 1]; ++k)
        mipmap.setAt(row + g.dir_C[k] / compressionRatio);
    }
  }
};

}  // namespace kites

#endif
