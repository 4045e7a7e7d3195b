// ref_harness.cpp -- runs farkhor/KiTES's OWN host code, compiled from the
// reference headers where they lie (see oracle/Makefile), as the pinned
// oracle and the reference CPU baseline.  TEST INFRASTRUCTURE ONLY.
//
// Modes
//   build <edgelist> <vpg> <sd|ds> <source> <sssp|label> <dir|undir> <out>
//       kites::graph_csr<unsigned,unsigned> from an edge-list file with a
//       pre-processing function of the same form as the reference example's
//       (examples/sssp_basic_single_device.cu:9-27), then the reference's
//       kites::sanity_check raw overload (kites/graph/sanity_check.cuh:13-59)
//       over the built arrays.  Dumps every public member of the host graph
//       plus the fixed point and the sweep count.
//   mipmap <edgelist> <cr> <sd|ds> <source> <out>
//       kites::graph_csr_mipmapped<unsigned,unsigned> with compression
//       ratio cr from an edge-list file and the same pre-processing
//       function (SSSP values); dumps V, R, C, E, the block frontier and the
//       block mipmap (kites/graph/graph_csr_mipmapped.hpp:40-78).
//   save <edgelist> <vpg> <source> <out>
//       the directed kites::graph_csr of `build` (SSSP values) written in the
//       reference's prepared text format by kites::io::save_to_file
//       (kites/io/graph_output.cuh:23-31).
//   csc <in> <sssp_wrap|sssp_sat|bfs|cc> <out> [max_seconds]
//       Reads a binary CSC and runs the reference's sanity_check loop on it
//       with the four user functions of the chosen operator; dumps V and the
//       wall time of the loop.
//
// The functions below are this harness's own; the graph construction and
// the fixed-point loop are the reference's code, included unmodified.
#include "kites/graph/sanity_check.cuh"
#include "kites/graph/graph_csr_mipmapped.hpp"
#include "kites/io/graph_output.cuh"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

unsigned g_source = 0;
unsigned g_inf = 1073741823u;
bool g_label_init = false;

// Same contract as the reference example's pre-processing function:
// set both endpoint values, set the edge value (third column if present,
// else (s+1)(d+2) % 127), return whether the destination starts active.
template <typename vT, class eT>
bool harness_preprocess(const unsigned int argcount, char **argvector,
                        const unsigned int s, const unsigned int d, vT &sv,
                        vT &dv, eT &e) {
  if (g_label_init) {
    sv = s;
    dv = d;
  } else {
    sv = (s == g_source) ? 0 : g_inf;
    dv = (d == g_source) ? 0 : g_inf;
  }
  e = (argcount > 0) ? static_cast<eT>(atoi(argvector[0]))
                     : static_cast<eT>((s + 1) * (d + 2) % 127);
  return g_label_init ? true : (s == g_source);
}

template <class T>
void put(FILE *f, const T *p, size_t n) {
  if (n && fwrite(p, sizeof(T), n, f) != n) {
    perror("fwrite");
    exit(3);
  }
}

template <class T>
void get(FILE *f, T *p, size_t n) {
  if (n && fread(p, sizeof(T), n, f) != n) {
    perror("fread");
    exit(3);
  }
}

int run_build(int argc, char **argv) {
  if (argc < 9) return 2;
  const char *path = argv[2];
  unsigned vpg = static_cast<unsigned>(atoi(argv[3]));
  bool sd = std::string(argv[4]) == "sd";
  g_source = static_cast<unsigned>(strtoul(argv[5], nullptr, 10));
  g_label_init = std::string(argv[6]) == "label";
  bool directed = std::string(argv[7]) == "dir";
  const char *out = argv[8];
  if (argc > 9) g_inf = static_cast<unsigned>(strtoul(argv[9], nullptr, 10));
  auto form = sd ? kites::input_graph_form::edge_list_s_d
                 : kites::input_graph_form::edge_list_d_s;

  using vT = unsigned;
  using eT = unsigned;
  auto initF = [](volatile vT &l, vT &g) { l = g; };
  auto compWrap = [](volatile vT &p, vT s, eT *w) { p = s + *w; };
  auto compLabel = [](volatile vT &p, vT s, eT *) { p = s; };
  auto redF = [](volatile vT &l, volatile vT &r) { if (l > r) l = r; };
  auto updF = [](volatile vT &n, vT o) { return n < o; };

  auto dump_and_check = [&](kites::graph_csr<vT, eT> &g) {
    FILE *f = fopen(out, "wb");
    if (!f) { perror(out); exit(3); }
    uint64_t hdr[8] = {g.get_num_vertices(), g.get_num_edges(),
                       g.vBitmap.getnBits(), g.vBitmap.size(),
                       g.dir_R.size(), g.dir_C.size(),
                       g.gProp == kites::graph_property::directed ? 1u : 0u,
                       g.getVertexPerGroup()};
    put(f, hdr, 8);
    put(f, g.V.get_ptr(), g.V.size());
    put(f, g.R.get_ptr(), g.R.size());
    put(f, g.C.get_ptr(), g.C.size());
    put(f, g.E.get_ptr(), g.E.size());
    put(f, g.vBitmap.get_ptr(), g.vBitmap.size());
    put(f, g.dir_R.get_ptr(), g.dir_R.size());
    put(f, g.dir_C.get_ptr(), g.dir_C.size());
    // The reference's fixed point over a copy of the initial values.
    const kites::uva_buffer<vT> &initial = g.V;
    kites::host_pinned_buffer<vT> Vfix(initial);
    kites::host_pinned_buffer<vT> cmp(initial);
    if (g_label_init)
      kites::sanity_check(g.get_num_vertices(), Vfix, g.R, g.C, g.E, cmp,
                          initF, compLabel, redF, updF);
    else
      kites::sanity_check(g.get_num_vertices(), Vfix, g.R, g.C, g.E, cmp,
                          initF, compWrap, redF, updF);
    put(f, Vfix.get_ptr(), Vfix.size());
    fclose(f);
  };

  if (directed) {
    kites::graph_csr<vT, eT> g(path, harness_preprocess<vT, eT>, vpg, form);
    dump_and_check(g);
  } else {
    kites::graph_csr<vT, eT> g(path, harness_preprocess<vT, eT>, form,
                               kites::graph_property::undirected,
                               kites::edge_list_expression::incomplete);
    dump_and_check(g);
  }
  return 0;
}

int run_mipmap(int argc, char **argv) {
  if (argc < 7) return 2;
  const char *path = argv[2];
  const unsigned cr = static_cast<unsigned>(atoi(argv[3]));
  const bool sd = std::string(argv[4]) == "sd";
  g_source = static_cast<unsigned>(strtoul(argv[5], nullptr, 10));
  g_label_init = false;
  const char *out = argv[6];
  using vT = unsigned;
  using eT = unsigned;
  kites::graph_csr_mipmapped<vT, eT> g(
      path, harness_preprocess<vT, eT>, cr,
      sd ? kites::input_graph_form::edge_list_s_d : kites::input_graph_form::edge_list_d_s);
  FILE *f = fopen(out, "wb");
  if (!f) { perror(out); exit(3); }
  uint64_t hdr[6] = {g.get_num_vertices(), g.get_num_edges(), g.compressionRatio,
                     g.mipmapDim, g.vBitmap.size(), g.mipmap.size()};
  put(f, hdr, 6);
  put(f, g.V.get_ptr(), g.V.size());
  put(f, g.R.get_ptr(), g.R.size());
  put(f, g.C.get_ptr(), g.C.size());
  put(f, g.E.get_ptr(), g.E.size());
  put(f, g.vBitmap.get_ptr(), g.vBitmap.size());
  put(f, g.mipmap.get_ptr(), g.mipmap.size());
  fclose(f);
  return 0;
}

int run_save(int argc, char **argv) {
  if (argc < 6) return 2;
  const unsigned vpg = static_cast<unsigned>(atoi(argv[3]));
  g_source = static_cast<unsigned>(strtoul(argv[4], nullptr, 10));
  g_label_init = false;
  kites::graph_csr<unsigned, unsigned> g(argv[2], harness_preprocess<unsigned, unsigned>, vpg,
                                         kites::input_graph_form::edge_list_s_d);
  kites::io::save_to_file(g, std::string(argv[5]));
  return 0;
}

int run_csc(int argc, char **argv) {
  if (argc < 5) return 2;
  std::string op = argv[3];
  FILE *f = fopen(argv[2], "rb");
  if (!f) { perror(argv[2]); return 3; }
  uint64_t hdr[2];
  get(f, hdr, 2);
  const size_t n = hdr[0], m = hdr[1];
  using vT = unsigned;
  using eT = unsigned;
  kites::host_pinned_buffer<vT> V(n), Vcopy(n);
  kites::host_pinned_buffer<unsigned> R(n + 1), C(m);
  kites::host_pinned_buffer<eT> E(m);
  get(f, V.get_ptr(), n);
  get(f, R.get_ptr(), n + 1);
  get(f, C.get_ptr(), m);
  get(f, E.get_ptr(), m);
  fclose(f);
  std::memcpy(Vcopy.get_ptr(), V.get_ptr(), n * sizeof(vT));

  auto initF = [](volatile vT &l, vT &g) { l = g; };
  auto redF = [](volatile vT &l, volatile vT &r) { if (l > r) l = r; };
  auto updF = [](volatile vT &nv, vT o) { return nv < o; };
  auto t0 = std::chrono::steady_clock::now();
  if (op == "sssp_wrap") {
    auto c = [](volatile vT &p, vT s, eT *w) { p = s + *w; };
    kites::sanity_check(n, V, R, C, E, Vcopy, initF, c, redF, updF);
  } else if (op == "sssp_sat") {
    auto c = [](volatile vT &p, vT s, eT *w) {
      vT t = s + *w;
      p = (t < s) ? 0xFFFFFFFFu : t;
    };
    kites::sanity_check(n, V, R, C, E, Vcopy, initF, c, redF, updF);
  } else if (op == "bfs") {
    auto c = [](volatile vT &p, vT s, eT *) {
      p = (s == 0xFFFFFFFFu) ? 0xFFFFFFFFu : s + 1u;
    };
    kites::sanity_check(n, V, R, C, E, Vcopy, initF, c, redF, updF);
  } else if (op == "cc") {
    auto c = [](volatile vT &p, vT s, eT *) { p = s; };
    kites::sanity_check(n, V, R, C, E, Vcopy, initF, c, redF, updF);
  } else {
    fprintf(stderr, "unknown op %s\n", op.c_str());
    return 2;
  }
  auto t1 = std::chrono::steady_clock::now();
  double secs = std::chrono::duration<double>(t1 - t0).count();
  FILE *o = fopen(argv[4], "wb");
  if (!o) { perror(argv[4]); return 3; }
  put(o, &secs, 1);
  put(o, V.get_ptr(), n);
  fclose(o);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  try {
    if (argc >= 2 && std::string(argv[1]) == "build") return run_build(argc, argv);
    if (argc >= 2 && std::string(argv[1]) == "csc") return run_csc(argc, argv);
    if (argc >= 2 && std::string(argv[1]) == "mipmap") return run_mipmap(argc, argv);
    if (argc >= 2 && std::string(argv[1]) == "save") return run_save(argc, argv);
  } catch (const std::exception &e) {
    fprintf(stderr, "%s\n", e.what());
    return 4;
  }
  fprintf(stderr,
          "usage: ref_harness build <edges> <vpg> <sd|ds> <src> <sssp|label> "
          "<dir|undir> <out> [inf]\n"
          "       ref_harness csc <in> <sssp_wrap|sssp_sat|bfs|cc> <out>\n");
  return 2;
}

// ---- shared-library entry for bench.py's CPU baseline ----------------------
// Runs the reference's sanity_check loop (sanity_check.cuh:13-59) over
// caller arrays (copied into the reference's own host buffers), with the
// saturating SSSP / BFS / CC user functions; V is updated in place.
// Returns the loop's wall seconds, or a negative value on error.
extern "C" double ref_sanity_check_csc(int op, uint64_t n, uint64_t m,
                                       uint32_t *V_io, const uint32_t *R,
                                       const uint32_t *C, const uint32_t *E) {
  using vT = unsigned;
  using eT = unsigned;
  try {
    kites::host_pinned_buffer<vT> V(n), Vcopy(n);
    kites::host_pinned_buffer<unsigned> Rb(n + 1), Cb(m ? m : 1);
    kites::host_pinned_buffer<eT> Eb(m ? m : 1);
    std::memcpy(V.get_ptr(), V_io, n * sizeof(vT));
    std::memcpy(Vcopy.get_ptr(), V_io, n * sizeof(vT));
    std::memcpy(Rb.get_ptr(), R, (n + 1) * sizeof(unsigned));
    if (m) std::memcpy(Cb.get_ptr(), C, m * sizeof(unsigned));
    if (m && E) std::memcpy(Eb.get_ptr(), E, m * sizeof(eT));
    auto initF = [](volatile vT &l, vT &g) { l = g; };
    auto redF = [](volatile vT &l, volatile vT &r) { if (l > r) l = r; };
    auto updF = [](volatile vT &nv, vT o) { return nv < o; };
    auto t0 = std::chrono::steady_clock::now();
    if (op == 0) {
      auto c = [](volatile vT &p, vT s, eT *w) {
        vT t = s + *w;
        p = (t < s) ? 0xFFFFFFFFu : t;
      };
      kites::sanity_check(n, V, Rb, Cb, Eb, Vcopy, initF, c, redF, updF);
    } else if (op == 1) {
      auto c = [](volatile vT &p, vT s, eT *) {
        p = (s == 0xFFFFFFFFu) ? 0xFFFFFFFFu : s + 1u;
      };
      kites::sanity_check(n, V, Rb, Cb, Eb, Vcopy, initF, c, redF, updF);
    } else {
      auto c = [](volatile vT &p, vT s, eT *) { p = s; };
      kites::sanity_check(n, V, Rb, Cb, Eb, Vcopy, initF, c, redF, updF);
    }
    auto t1 = std::chrono::steady_clock::now();
    std::memcpy(V_io, V.get_ptr(), n * sizeof(vT));
    return std::chrono::duration<double>(t1 - t0).count();
  } catch (...) {
    return -1.0;
  }
}

// ---- many sources on all host threads (bench.py's reference arm) ----------
// SSSP (saturating add, the engine's KITES_OP_SSSP) from each of `n_sources`
// sources over one graph, each by the reference's own sanity_check loop
// (sanity_check.cuh:13-59), which is single-threaded: `threads` host threads
// take sources one at a time and run their loops side by side, sharing one
// copy of R, C and E in the reference's host buffers.  For source i,
// reached_edges[i] = the sum of out_degree over the vertices it reaches and
// secs_each[i] the wall seconds of its loop; dist_out (n x n_sources, column
// i at dist_out + i * n) may be NULL.  Returns the wall seconds from the
// first loop's start to the last one's end, or a negative value on error.
#include <atomic>
#include <thread>

extern "C" double ref_sssp_sources(uint64_t n, uint64_t m, const uint32_t *R,
                                   const uint32_t *C, const uint32_t *E,
                                   const uint32_t *sources, uint32_t n_sources,
                                   uint32_t threads, const uint64_t *out_degree,
                                   uint64_t *reached_edges, double *secs_each,
                                   uint32_t *dist_out) {
  using vT = unsigned;
  using eT = unsigned;
  try {
    if (m >= 0x80000000ull) return -2.0;  // the loop masks bit 31 of offsets
    kites::host_pinned_buffer<unsigned> Rb(n + 1), Cb(m ? m : 1);
    kites::host_pinned_buffer<eT> Eb(m ? m : 1);
    std::memcpy(Rb.get_ptr(), R, (n + 1) * sizeof(unsigned));
    if (m) std::memcpy(Cb.get_ptr(), C, m * sizeof(unsigned));
    if (m && E) std::memcpy(Eb.get_ptr(), E, m * sizeof(eT));
    std::atomic<uint32_t> next{0};
    std::atomic<bool> failed{false};
    auto worker = [&]() {
      try {
        kites::host_pinned_buffer<vT> V(n), Vcopy(n);
        for (uint32_t i; (i = next.fetch_add(1)) < n_sources;) {
          const uint32_t s = sources[i];
          for (uint64_t v = 0; v < n; ++v) V[v] = 0xFFFFFFFFu;
          V[s] = 0u;
          std::memcpy(Vcopy.get_ptr(), V.get_ptr(), n * sizeof(vT));
          auto initF = [](volatile vT &l, vT &g) { l = g; };
          auto redF = [](volatile vT &l, volatile vT &r) { if (l > r) l = r; };
          auto updF = [](volatile vT &nv, vT o) { return nv < o; };
          auto comp = [](volatile vT &p, vT sv, eT *w) {
            vT t = sv + *w;
            p = (t < sv) ? 0xFFFFFFFFu : t;
          };
          auto t0 = std::chrono::steady_clock::now();
          kites::sanity_check(n, V, Rb, Cb, Eb, Vcopy, initF, comp, redF, updF);
          auto t1 = std::chrono::steady_clock::now();
          if (secs_each) secs_each[i] = std::chrono::duration<double>(t1 - t0).count();
          if (reached_edges && out_degree) {
            uint64_t r = 0;
            for (uint64_t v = 0; v < n; ++v)
              if (V[v] != 0xFFFFFFFFu) r += out_degree[v];
            reached_edges[i] = r;
          }
          if (dist_out) std::memcpy(dist_out + (uint64_t)i * n, V.get_ptr(), n * sizeof(vT));
        }
      } catch (...) {
        failed = true;
      }
    };
    const uint32_t nt = std::max<uint32_t>(1, std::min(threads, n_sources));
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < nt; ++t) pool.emplace_back(worker);
    for (auto &th : pool) th.join();
    auto t1 = std::chrono::steady_clock::now();
    if (failed) return -1.0;
    return std::chrono::duration<double>(t1 - t0).count();
  } catch (...) {
    return -1.0;
  }
}
