// sssp_mipmapped.cu -- single-source shortest paths over a mipmapped graph
// (blocks of `cr` vertices, coarse activation through the block mipmap),
// then the CPU sanity check over the same CSC.
// Usage: sssp_mipmapped <edges> <source> <cr> [out_prefix]
//   out_prefix.bits / .mip: the host graph's block frontier and mipmap
//   (32-bit words, binary); out_prefix.dist: the device distances, one per
//   line.
// Build: nvcc -std=c++17 -O3 --expt-extended-lambda
//        -gencode arch=compute_100a,code=sm_100a -I include
//        examples/sssp_mipmapped.cu -L kites_b200 -lkites_b200
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>

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

static void write_words(const std::string &path, const kites::host_bitmap &b) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot open " + path);
  const std::size_t n = b.size();
  const bool ok = n == 0 || std::fwrite(b.get_ptr(), sizeof(unsigned), n, f) == n;
  std::fclose(f);
  if (!ok) throw std::runtime_error("short write to " + path);
}

int main(int argc, char **argv) {
  if (argc < 4) {
    std::cerr << "usage: " << argv[0] << " <edges> <source> <cr> [out_prefix]\n";
    return 2;
  }
  try {
    using vT = unsigned int;
    using eT = unsigned int;
    g_source = (unsigned)std::atoi(argv[2]);
    const unsigned cr = (unsigned)std::atoi(argv[3]);

    auto initF = [] __host__ __device__(volatile vT &loc, vT &glob) { loc = glob; };
    auto nbrCompF = [] __host__ __device__(volatile vT &partial, vT srcV, eT *e) {
      partial = srcV + *e;
    };
    auto redF = [] __host__ __device__(volatile vT &lhs, volatile vT &rhs) {
      if (lhs > rhs) lhs = rhs;
    };
    auto updF = [] __host__ __device__(volatile vT &nv, vT ov) { return nv < ov; };

    kites::graph_csr_mipmapped<vT, eT> host(argv[1], preprocess<vT, eT>, cr,
                                            kites::input_graph_form::edge_list_s_d);
    std::cout << "mipmapDim " << host.mipmapDim << "\n";
    kites::nv_gpu dev(0);
    auto dg = kites::make_graph_csr_for_device(host, dev);
    kites::process<kites::launch::sync>(dg, dev, initF, nbrCompF, redF, updF);
    if (argc > 4) {
      const std::string pre = argv[4];
      write_words(pre + ".bits", host.vBitmap);
      write_words(pre + ".mip", host.mipmap);
      kites::host_pinned_buffer<vT> result(dg.V);
      std::ofstream out(pre + ".dist");
      out << result;
    }
    const bool ok = kites::sanity_check(host, dg, initF, nbrCompF, redF, updF);
    return ok ? EXIT_SUCCESS : 3;
  } catch (const std::exception &e) {
    std::cerr << e.what() << "\nExiting." << std::endl;
    return EXIT_FAILURE;
  }
}
