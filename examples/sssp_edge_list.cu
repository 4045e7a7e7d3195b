// sssp_edge_list.cu -- single-source shortest paths over an edge-list file
// through the kites:: API (the drop-in for farkhor/KiTES), then the CPU
// sanity check.  Usage: sssp_edge_list <edges> [source] [vpg] [builtin] [out]
//   builtin = 1 runs the engine's precompiled SSSP instead of the lambdas;
//   out = file for the device distances, one per line.
// Build: nvcc -std=c++17 -O3 --expt-extended-lambda
//        -gencode arch=compute_100a,code=sm_100a -I include
//        examples/sssp_edge_list.cu -L kites_b200 -lkites_b200
#include <cstdlib>
#include <fstream>
#include <iostream>

#include "kites/kites.cuh"

static unsigned g_source = 0;

template <typename vT, class eT>
bool preprocess(const unsigned int argc, char **argv, const unsigned int s, const unsigned int d,
                vT &sv, vT &dv, eT &e) {
  const vT inf = 1073741823u;  // 2^30 - 1: distances stay far from wrap-around
  sv = (s == g_source) ? 0 : inf;
  dv = (d == g_source) ? 0 : inf;
  e = (argc > 0) ? static_cast<eT>(std::atoi(argv[0])) : static_cast<eT>((s * 7u + d * 13u) % 97u + 1u);
  return s == g_source;
}

int main(int argc, char **argv) {
  if (argc < 2) {
    std::cerr << "usage: " << argv[0] << " <edges> [source] [vpg] [builtin]\n";
    return 2;
  }
  try {
    using vT = unsigned int;
    using eT = unsigned int;
    g_source = argc > 2 ? (unsigned)std::atoi(argv[2]) : 0u;
    const unsigned vpg = argc > 3 ? (unsigned)std::atoi(argv[3]) : 1u;
    const bool builtin = argc > 4 && std::atoi(argv[4]) != 0;

    auto initF = [] __host__ __device__(volatile vT &loc, vT &glob) { loc = glob; };
    auto nbrCompF = [] __host__ __device__(volatile vT &partial, vT srcV, eT *e) {
      partial = srcV + *e;
    };
    auto redF = [] __host__ __device__(volatile vT &lhs, volatile vT &rhs) {
      if (lhs > rhs) lhs = rhs;
    };
    auto updF = [] __host__ __device__(volatile vT &nv, vT ov) { return nv < ov; };

    kites::graph_csr<vT, eT> host(argv[1], preprocess<vT, eT>, vpg,
                                  kites::input_graph_form::edge_list_s_d);
    kites::nv_gpu dev(0);
    auto dg = kites::make_graph_csr_for_device(host, dev);
    if (builtin) {
      auto st = kites::process<kites::launch::sync>(dg, dev, kites::ops::sssp_wrap);
      std::cout << "Engine: " << st.iterations << " iterations, " << st.device_ms << " ms\n";
    } else {
      kites::process<kites::launch::sync>(dg, dev, initF, nbrCompF, redF, updF);
    }
    if (argc > 5) {  // device distances, one per line
      kites::host_pinned_buffer<vT> result(dg.V);
      std::ofstream out(argv[5]);
      out << result;
    }
    const bool ok = kites::sanity_check(host, dg, initF, nbrCompF, redF, updF);
    return ok ? EXIT_SUCCESS : 3;
  } catch (const std::exception &e) {
    std::cerr << e.what() << "\nExiting." << std::endl;
    return EXIT_FAILURE;
  }
}
