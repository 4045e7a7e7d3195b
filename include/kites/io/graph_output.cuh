// graph_output.cuh -- text output of vertex values and the prepared graph
// format read back by graph_csr(file) (farkhor/KiTES kites/io/graph_output.cuh:11-38):
// counts, directed flag, then V, R, C, E, vBitmap words [, dir_R, dir_C],
// one value per line.
#ifndef KITES_B200_GRAPH_OUTPUT_CUH_
#define KITES_B200_GRAPH_OUTPUT_CUH_

#include <fstream>
#include <string>

#include "../graph/graph_csr.h"
#include "file_interactor.hpp"

namespace kites {
namespace io {

template <class vT, class eT, class vIdxT>
void out_vertices(graph_csr<vT, eT, vIdxT> &g, std::ofstream &out) {
  out << g.V;
}

template <class vT, class eT, class vIdxT>
void out_vertices(graph_csr<vT, eT, vIdxT> &g, const std::string &file) {
  std::ofstream out;
  openFileToAccess(out, file);
  out_vertices(g, out);
}

template <class vT, class eT, class vIdxT>
void save_to_file(graph_csr<vT, eT, vIdxT> &g, std::ofstream &out) {
  out << g.get_num_vertices() << "\n" << g.get_num_edges() << "\n"
      << (g.gProp == graph_property::directed ? 1 : 0) << "\n";
  out << g.V << g.R << g.C << g.E << g.vBitmap;
  if (g.gProp == graph_property::directed) out << g.dir_R << g.dir_C;
}

template <class vT, class eT, class vIdxT>
void save_to_file(graph_csr<vT, eT, vIdxT> &g, const std::string &file) {
  std::ofstream out;
  openFileToAccess(out, file);
  save_to_file(g, out);
}

}  // namespace io
}  // namespace kites

#endif
