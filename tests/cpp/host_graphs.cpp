// host_graphs.cpp -- dumps what the kites:: host graph classes of
// include/kites/ build from an edge-list file, for comparison with the
// oracle and the golden hashes of the reference's own construction.
//   host_graphs csr <edges> <vpg> <source> <out>
//       kites::graph_csr<unsigned,unsigned>(file, f, vpg, edge_list_s_d):
//       V, R, C, E, vBitmap words, dir_R, dir_C.
//   host_graphs undir <edges> 1 <source> <out>
//       kites::graph_csr<unsigned,unsigned>(file, f, edge_list_s_d, undirected,
//       incomplete): the same arrays (dir_R, dir_C empty).
//   host_graphs save <edges> <vpg> <source> <out>
//       kites::io::save_to_file of the directed graph_csr (prepared text).
//   host_graphs load <prepared> 1 <source> <out>
//       kites::graph_csr<unsigned,unsigned>(prepared file): the csr arrays.
//   host_graphs check <edges> <vpg> <source> <values>
//       kites::sanity_check over the directed graph_csr with the reference
//       example's four functions (wrap-around add, min, less-than) against
//       the uint32 values in the binary file <values>; exit status 0 iff it
//       passes (its report goes to stdout).
//   host_graphs mip <edges> <cr> <source> <out>
//       kites::graph_csr_mipmapped<unsigned,unsigned>(file, f, cr):
//       V, R, C, E, vBitmap words, mipmap words.
// The pre-processing function is the reference example's (values 0 at the
// source and 2^30 - 1 elsewhere, the edge value from the third column or
// (s + 1)(d + 2) % 127, the destination active iff the source is `source`).
// Each dump starts with the element counts as uint64.  Test infrastructure.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "kites/graph/graph_csr.h"
#include "kites/graph/graph_csr_mipmapped.hpp"
#include "kites/graph/sanity_check.cuh"
#include "kites/io/graph_output.cuh"

namespace {

unsigned g_source = 0;

template <typename vT, class eT>
bool preprocess(const unsigned int argc, char **argv, const unsigned int s, const unsigned int d,
                vT &sv, vT &dv, eT &e) {
  const vT inf = 1073741823u;
  sv = (s == g_source) ? 0 : inf;
  dv = (d == g_source) ? 0 : inf;
  e = (argc > 0) ? static_cast<eT>(std::atoi(argv[0])) : static_cast<eT>((s + 1) * (d + 2) % 127);
  return s == g_source;
}

template <class T>
void put(FILE *f, const T *p, size_t n) {
  if (n && std::fwrite(p, sizeof(T), n, f) != n) std::exit(3);
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 6) return 2;
  const std::string mode = argv[1];
  const unsigned param = static_cast<unsigned>(std::atoi(argv[3]));
  g_source = static_cast<unsigned>(std::strtoul(argv[4], nullptr, 10));
  if (mode == "check") {
    try {
      kites::graph_csr<unsigned, unsigned> g(argv[2], preprocess<unsigned, unsigned>, param,
                                             kites::input_graph_form::edge_list_s_d);
      kites::host_pinned_buffer<unsigned> want(g.get_num_vertices());
      FILE *vf = std::fopen(argv[5], "rb");
      if (!vf) return 3;
      const size_t got = std::fread(want.get_ptr(), sizeof(unsigned), want.size(), vf);
      std::fclose(vf);
      if (got != want.size()) return 3;
      auto initF = [](unsigned &loc, unsigned &glob) { loc = glob; };
      auto compF = [](unsigned &partial, unsigned srcV, unsigned *e) { partial = srcV + *e; };
      auto redF = [](unsigned &lhs, unsigned &rhs) { if (lhs > rhs) lhs = rhs; };
      auto updF = [](unsigned &nv, unsigned ov) { return nv < ov; };
      const bool ok = kites::sanity_check(g.get_num_vertices(), g.V, g.R, g.C, g.E, want, initF,
                                          compF, redF, updF);
      return ok ? 0 : 5;
    } catch (const std::exception &e) {
      std::fprintf(stderr, "%s\n", e.what());
      return 4;
    }
  }
  if (mode == "save") {
    try {
      kites::graph_csr<unsigned, unsigned> g(argv[2], preprocess<unsigned, unsigned>, param,
                                             kites::input_graph_form::edge_list_s_d);
      kites::io::save_to_file(g, std::string(argv[5]));
    } catch (const std::exception &e) {
      std::fprintf(stderr, "%s\n", e.what());
      return 4;
    }
    return 0;
  }
  FILE *f = std::fopen(argv[5], "wb");
  if (!f) return 3;
  try {
    if (mode == "csr" || mode == "undir" || mode == "load") {
      kites::graph_csr<unsigned, unsigned> g =
          mode == "load" ? kites::graph_csr<unsigned, unsigned>(std::string(argv[2]))
          : mode == "csr"
              ? kites::graph_csr<unsigned, unsigned>(argv[2], preprocess<unsigned, unsigned>, param,
                                                     kites::input_graph_form::edge_list_s_d)
              : kites::graph_csr<unsigned, unsigned>(argv[2], preprocess<unsigned, unsigned>,
                                                     kites::input_graph_form::edge_list_s_d,
                                                     kites::graph_property::undirected,
                                                     kites::edge_list_expression::incomplete);
      const uint64_t hdr[7] = {g.V.size(), g.R.size(), g.C.size(), g.E.size(),
                               g.vBitmap.size(), g.dir_R.size(), g.dir_C.size()};
      put(f, hdr, 7);
      put(f, g.V.get_ptr(), g.V.size());
      put(f, g.R.get_ptr(), g.R.size());
      put(f, g.C.get_ptr(), g.C.size());
      put(f, g.E.get_ptr(), g.E.size());
      put(f, g.vBitmap.get_ptr(), g.vBitmap.size());
      put(f, g.dir_R.get_ptr(), g.dir_R.size());
      put(f, g.dir_C.get_ptr(), g.dir_C.size());
    } else {
      kites::graph_csr_mipmapped<unsigned, unsigned> g(argv[2], preprocess<unsigned, unsigned>,
                                                       param);
      const uint64_t hdr[7] = {g.V.size(), g.R.size(), g.C.size(), g.E.size(),
                               g.vBitmap.size(), g.mipmap.size(), g.mipmapDim};
      put(f, hdr, 7);
      put(f, g.V.get_ptr(), g.V.size());
      put(f, g.R.get_ptr(), g.R.size());
      put(f, g.C.get_ptr(), g.C.size());
      put(f, g.E.get_ptr(), g.E.size());
      put(f, g.vBitmap.get_ptr(), g.vBitmap.size());
      put(f, g.mipmap.get_ptr(), g.mipmap.size());
    }
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    std::fclose(f);
    return 4;
  }
  std::fclose(f);
  return 0;
}
