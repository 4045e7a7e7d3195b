// sssp_binary_csc.cu -- SSSP through kites::process with user functions on
// a graph read from a binary CSC file: the drop-in API path timed on large
// graphs.
//
//   sssp_binary_csc <graph.csc> <source> [<source> ...] [--dump <file>]
//
// The four functions are those of the reference's example
// (examples/sssp_basic_single_device.cu:40-47), and so are the initial
// values: V = 2^30 - 1 except V[source] = 0, the frontier the source's
// out-neighbours.  The graph is uploaded once; for every source the values
// and frontier are reset on the device and kites::process runs.  One JSON
// line per source: iterations, the loop's device time (CUDA events), the
// edges whose source endpoint is reached and a 64-bit FNV-1a digest of the
// distances; --dump writes the last source's distances (uint32, raw).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "kites/kites.cuh"

int main(int argc, char **argv) {
  if (argc < 3) {
    std::cerr << "usage: " << argv[0] << " <graph.csc> <source> [<source> ...] [--dump file]\n";
    return 2;
  }
  try {
    using vT = unsigned int;
    using eT = unsigned int;
    const vT kInf = 1073741823u;
    std::vector<unsigned> sources;
    std::string dump;
    for (int i = 2; i < argc; ++i) {
      if (std::string(argv[i]) == "--dump" && i + 1 < argc) {
        dump = argv[++i];
        continue;
      }
      sources.push_back((unsigned)std::strtoul(argv[i], nullptr, 10));
    }
    auto initF = [] __host__ __device__(volatile vT &locV, vT &globV) { locV = globV; };
    auto nbrCompF = [] __host__ __device__(volatile vT &partialV, vT srcV, eT *connE) {
      partialV = srcV + (*connE);
    };
    auto redF = [] __host__ __device__(volatile vT &lhsV, volatile vT &rhsV) {
      if (lhsV > rhsV) lhsV = rhsV;
    };
    auto updF = [] __host__ __device__(volatile vT &newV, vT oldV) { return newV < oldV; };

    kites::graph_csr<vT, eT> h(argv[1], kites::io::binary_csc);
    const std::size_t n = h.get_num_vertices(), m = h.get_num_edges();
    // Out-degrees (the reached-edge count) and, per source, its
    // out-neighbours (the first frontier).
    std::vector<uint64_t> outdeg(n, 0);
    for (std::size_t e = 0; e < m; ++e) ++outdeg[h.C[e]];
    kites::nv_gpu dev(0);
    for (std::size_t v = 0; v < n; ++v) h.V[v] = kInf;
    auto d = kites::make_graph_csr_for_device(h, dev);
    std::vector<vT> V(n), init(n);
    std::vector<uint32_t> bits((n + 31) / 32);
    for (unsigned src : sources) {
      if (src >= n) throw std::runtime_error("source out of range");
      std::fill(init.begin(), init.end(), kInf);
      init[src] = 0;
      std::fill(bits.begin(), bits.end(), 0u);
      for (std::size_t v = 0; v < n; ++v)
        for (unsigned e = h.R[v]; e < h.R[v + 1]; ++e)
          if (h.C[e] == src) bits[v >> 5] |= 1u << (v & 31);
      KITESErrorCheck(kites_graph_set_values(d.engine_graph(), init.data(), n));
      KITESErrorCheck(kites_graph_set_frontier(d.engine_graph(), bits.data(), n));
      kites::process<kites::launch::sync>(d, dev, initF, nbrCompF, redF, updF);
      KITESErrorCheck(kites_graph_get_values(d.engine_graph(), V.data(), n));
      uint64_t reached = 0, h64 = 1469598103934665603ull;
      for (std::size_t v = 0; v < n; ++v) {
        if (V[v] != kInf) reached += outdeg[v];
        for (int b = 0; b < 4; ++b) {
          h64 ^= (V[v] >> (8 * b)) & 0xFFu;
          h64 *= 1099511628211ull;
        }
      }
      std::printf("{\"source\": %u, \"iterations\": %llu, \"device_ms\": %.4f, "
                  "\"reached_edges\": %llu, \"digest\": \"%016llx\"}\n",
                  src, (unsigned long long)d.last_iterations, d.last_device_ms,
                  (unsigned long long)reached, (unsigned long long)h64);
    }
    if (!dump.empty()) {
      FILE *f = std::fopen(dump.c_str(), "wb");
      if (!f || std::fwrite(V.data(), sizeof(vT), n, f) != n)
        throw std::runtime_error("cannot write " + dump);
      std::fclose(f);
    }
    return 0;
  } catch (const std::exception &e) {
    std::cerr << e.what() << "\n";
    return 1;
  }
}
