// graph_csr.h -- the host graph of the kites:: API (farkhor/KiTES
// kites/graph/graph_csr.h:21-232 with kites/graph/graph_raw.h:57-190).
//
// Construction rules kept from the reference (they fix the results):
//  * lines whose first character is not a digit are skipped; the first two
//    space/tab separated fields are vertex indices, any further fields are
//    handed to the pre-processing function as (argc, argv);
//  * the pre-processing function sets both endpoint values and the edge
//    value and returns whether the destination (group) starts active;
//    vertices that never appear keep a value-initialised vT;
//  * the CSC is keyed by destination, each row sorted by source (ties in
//    file order);
//  * directed graphs get the out-adjacency dir_R/dir_C: for vpg == 1 the
//    destinations of each source in ascending order, for vpg > 1 the sorted
//    distinct destination groups of each source group;
//  * V is padded to a multiple of 128 with empty rows; for directed vpg == 1
//    graphs the frontier bitmap and dir_R cover the padded range;
//  * an undirected graph gets no out-adjacency and, as in the reference, no
//    initial frontier bits.
#ifndef KITES_B200_GRAPH_CSR_H_
#define KITES_B200_GRAPH_CSR_H_

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <string>
#include <vector>

#include "../../kites_b200.h"
#include "../common/cuda_error_check.cuh"
#include "../common/globals.cuh"
#include "../io/file_interactor.hpp"
#include "../memory/host_pinned_buffer.cuh"
#include "graph_base.h"

namespace kites {

namespace io {
// Selects the binary CSC constructor of graph_csr (files written by
// kites_csc_save; no counterpart in the reference, whose only on-disk form
// of a built graph is the prepared text format).
struct binary_csc_t {};
constexpr binary_csc_t binary_csc{};
}  // namespace io

template <class vT, class eT, class vIdxT = unsigned int>
class graph_csr : public graph_base {
 public:
  using eIdxT = vIdxT;

  host_pinned_buffer<vT> V;
  host_pinned_buffer<eIdxT> R;
  host_pinned_buffer<vIdxT> C;
  host_pinned_buffer<eT> E;
  host_bitmap vBitmap;
  host_pinned_buffer<unsigned int> updateFlag;
  graph_property gProp;
  unsigned int vertexPerGroup;
  host_pinned_buffer<eIdxT> dir_R;
  host_pinned_buffer<vIdxT> dir_C;

  unsigned int getVertexPerGroup() const { return vertexPerGroup; }

  template <class funcT>
  graph_csr(std::ifstream &in, funcT f, input_graph_form gForm = input_graph_form::edge_list_s_d,
            graph_property gPropIn = graph_property::directed,
            edge_list_expression elExp = edge_list_expression::complete)
      : gProp{gPropIn}, vertexPerGroup{1} {
    construct(in, f, 1, gForm, gProp, elExp);
  }
  template <class funcT>
  graph_csr(const std::string &file, funcT f,
            input_graph_form gForm = input_graph_form::edge_list_s_d,
            graph_property gPropIn = graph_property::directed,
            edge_list_expression elExp = edge_list_expression::complete)
      : gProp{gPropIn}, vertexPerGroup{1} {
    std::ifstream in;
    io::openFileToAccess(in, file);
    construct(in, f, 1, gForm, gProp, elExp);
  }
  // The vertex-grouping constructors always build a directed graph
  // (graph_csr.h:210-230).
  template <class funcT>
  graph_csr(std::ifstream &in, funcT f, unsigned int vpg,
            input_graph_form gForm = input_graph_form::edge_list_s_d)
      : gProp{graph_property::directed}, vertexPerGroup{vpg} {
    construct(in, f, vpg, gForm, gProp, edge_list_expression::complete);
  }
  template <class funcT>
  graph_csr(const std::string &file, funcT f, unsigned int vpg,
            input_graph_form gForm = input_graph_form::edge_list_s_d)
      : gProp{graph_property::directed}, vertexPerGroup{vpg} {
    std::ifstream in;
    io::openFileToAccess(in, file);
    construct(in, f, vpg, gForm, gProp, edge_list_expression::complete);
  }
  // The prepared format written by io::save_to_file (graph_csr.h:112-166).
  explicit graph_csr(std::ifstream &in) : vertexPerGroup{1} { construct_prepared(in); }
  explicit graph_csr(const std::string &file) : vertexPerGroup{1} {
    std::ifstream in;
    io::openFileToAccess(in, file);
    construct_prepared(in);
  }
  // A binary CSC file (kites_csc_save): R, C and E as stored, rows padded to
  // a multiple of 128, V value-initialised and no frontier bit set -- the
  // caller sets V and vBitmap, as a pre-processing function would, before
  // uploading.  Directed graphs get no dir_R / dir_C here: the upload
  // derives the out-adjacency from the CSC (vertex_per_group 1).
  graph_csr(const std::string &file, io::binary_csc_t) : vertexPerGroup{1} {
    static_assert(sizeof(vIdxT) == 4, "binary CSC files hold 32-bit indices");
    uint64_t n = 0, m = 0;
    int has_e = 0, directed = 0;
    KITESErrorCheck(kites_csc_info(file.c_str(), &n, &m, &has_e, &directed, nullptr, 0));
    if (m > 0xFFFFFFFFull) throw std::runtime_error("graph_csr takes < 2^32 edges");
    std::vector<uint64_t> R64(n + 1);
    const std::size_t n_pad = (n % 128) ? (n / 128 + 1) * 128 : n;
    set_num_vertices(n_pad);
    set_num_edges(m);
    V.alloc(n_pad);
    R.alloc(n_pad + 1);
    C.alloc(m);
    E.alloc(m);
    updateFlag.alloc(1);
    updateFlag[0] = 0;
    std::vector<uint32_t> E32;
    const bool direct_e = sizeof(eT) == 4;
    if (has_e && !direct_e) E32.resize(m);
    KITESErrorCheck(kites_csc_load(file.c_str(), R64.data(), reinterpret_cast<uint32_t *>(C.get_ptr()),
                                   has_e ? (direct_e ? reinterpret_cast<uint32_t *>(E.get_ptr())
                                                     : E32.data())
                                         : nullptr));
    for (std::size_t v = 0; v <= n_pad; ++v) R[v] = static_cast<eIdxT>(R64[v < n ? v : n]);
    if (has_e && !direct_e)
      for (std::size_t i = 0; i < m; ++i) E[i] = static_cast<eT>(E32[i]);
    if (!has_e)
      for (std::size_t i = 0; i < m; ++i) E[i] = eT();
    for (std::size_t v = 0; v < n_pad; ++v) V[v] = vT();
    gProp = directed ? graph_property::directed : graph_property::undirected;
    vBitmap.alloc(n_pad);
    vBitmap.reset();
  }

 private:
  struct raw_edge {
    vIdxT dst, src;
    eT val;
    std::size_t order;
  };

  static bool split_fields(const std::string &line, std::vector<char> &buf,
                           std::vector<char *> &fields) {
    buf.assign(line.begin(), line.end());
    buf.push_back('\0');
    fields.clear();
    char *p = buf.data();
    while (*p) {
      while (*p == ' ' || *p == '\t') ++p;
      if (!*p) break;
      char *start = p;
      while (*p && *p != ' ' && *p != '\t') ++p;
      if (*p) *p++ = '\0';
      fields.push_back(start);
    }
    return fields.size() >= 2;
  }

  template <class funcT>
  void construct(std::ifstream &in, funcT f, unsigned int vpg, input_graph_form gForm,
                 graph_property gp, edge_list_expression elExp) {
    if (vpg == 0 || (vpg & (vpg - 1)))
      throw std::runtime_error("vertex per group must be a power of two");
    std::vector<vT> vals(1, vT());            // the reference starts with one vertex
    std::vector<char> act(1, 0);              // per group
    std::vector<raw_edge> edges;
    std::string line;
    std::vector<char> buf;
    std::vector<char *> fields;
    std::size_t order = 0;
    while (std::getline(in, line)) {
      if (line.empty() || line[0] < '0' || line[0] > '9') continue;
      if (!split_fields(line, buf, fields)) continue;
      const vIdxT first = static_cast<vIdxT>(std::atoll(fields[0]));
      const vIdxT second = static_cast<vIdxT>(std::atoll(fields[1]));
      const vIdxT hi = std::max(first, second);
      const bool sd = gForm == input_graph_form::edge_list_s_d;
      const vIdxT s = sd ? first : second, d = sd ? second : first;
      if (vals.size() <= hi) {
        vals.resize((std::size_t)hi + 1, vT());
        act.resize(((std::size_t)hi + 1 + vpg - 1) / vpg, 0);
      }
      const unsigned int argc = (unsigned int)fields.size() - 2;
      char **argv = fields.data() + 2;
      eT ev{};
      if (f(argc, argv, s, d, vals[s], vals[d], ev)) act[d / vpg] = 1;
      edges.push_back({d, s, ev, order++});
      if (gp == graph_property::undirected && elExp == edge_list_expression::incomplete) {
        eT rv{};
        if (f(argc, argv, d, s, vals[d], vals[s], rv)) act[s / vpg] = 1;
        edges.push_back({s, d, rv, order++});
      }
    }
    const std::size_t n = vals.size();
    std::stable_sort(edges.begin(), edges.end(), [](const raw_edge &a, const raw_edge &b) {
      return a.dst != b.dst ? a.dst < b.dst : a.src < b.src;
    });
    const std::size_t m = edges.size();
    const std::size_t n_pad = (n % 128) ? (n / 128 + 1) * 128 : n;
    const std::size_t ngroups = (n + vpg - 1) / vpg;
    set_num_vertices(n_pad);
    set_num_edges(m);
    V.alloc(n_pad);
    R.alloc(n_pad + 1);
    C.alloc(m);
    E.alloc(m);
    updateFlag.alloc(1);
    updateFlag[0] = 0;
    for (std::size_t v = 0; v < n_pad; ++v) V[v] = v < n ? vals[v] : vT();
    std::size_t e = 0;
    for (std::size_t v = 0; v <= n_pad; ++v) {
      while (v > 0 && e < m && edges[e].dst < v) ++e;
      R[v] = static_cast<eIdxT>(e);
    }
    for (std::size_t i = 0; i < m; ++i) {
      C[i] = edges[i].src;
      E[i] = edges[i].val;
    }
    if (gp == graph_property::directed) {
      std::vector<std::pair<vIdxT, vIdxT>> out;  // (source group, destination group)
      out.reserve(m);
      for (std::size_t i = 0; i < m; ++i)
        out.emplace_back(edges[i].src / vpg, edges[i].dst / vpg);
      std::stable_sort(out.begin(), out.end());
      if (vpg != 1) out.erase(std::unique(out.begin(), out.end()), out.end());
      const std::size_t rows = (vpg == 1) ? n_pad : ngroups;
      dir_R.alloc(rows + 1);
      dir_C.alloc(out.size());
      std::size_t k = 0;
      for (std::size_t r = 0; r <= rows; ++r) {
        while (r > 0 && k < out.size() && out[k].first < r) ++k;
        dir_R[r] = static_cast<eIdxT>(k);
      }
      for (std::size_t i = 0; i < out.size(); ++i) dir_C[i] = out[i].second;
      const std::size_t nbits = (vpg == 1) ? n_pad : ngroups;
      vBitmap.alloc(nbits);
      vBitmap.reset();
      for (std::size_t gi = 0; gi < ngroups; ++gi)
        if (act[gi]) vBitmap.setAt(gi);
    } else {
      vBitmap.alloc(ngroups);
      vBitmap.reset();
    }
  }

  void construct_prepared(std::ifstream &in) {
    std::string line;
    std::getline(in, line);
    const std::size_t n = std::stoull(line);
    std::getline(in, line);
    const std::size_t m = std::stoull(line);
    std::getline(in, line);
    gProp = (std::stoi(line) == 1) ? graph_property::directed : graph_property::undirected;
    set_num_vertices(n);
    set_num_edges(m);
    V.alloc(n);
    R.alloc(n + 1);
    C.alloc(m);
    E.alloc(m);
    vBitmap.alloc(n);
    updateFlag.alloc(1);
    updateFlag[0] = 0;
    auto next = [&]() {
      std::getline(in, line);
      return std::stoull(line);
    };
    for (std::size_t i = 0; i < n; ++i) V[i] = static_cast<vT>(next());
    for (std::size_t i = 0; i <= n; ++i) R[i] = static_cast<eIdxT>(next());
    for (std::size_t i = 0; i < m; ++i) C[i] = static_cast<vIdxT>(next());
    for (std::size_t i = 0; i < m; ++i) E[i] = static_cast<eT>(next());
    for (std::size_t i = 0; i < vBitmap.size(); ++i) vBitmap[i] = static_cast<unsigned int>(next());
    if (gProp == graph_property::directed) {
      dir_R.alloc(n + 1);
      dir_C.alloc(m);
      for (std::size_t i = 0; i <= n; ++i) dir_R[i] = static_cast<eIdxT>(next());
      for (std::size_t i = 0; i < m; ++i) dir_C[i] = static_cast<vIdxT>(next());
    }
  }
};

}  // namespace kites

#endif
