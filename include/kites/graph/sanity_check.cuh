// sanity_check.cuh -- the CPU verifier of the kites:: API (farkhor/KiTES
// kites/graph/sanity_check.cuh:13-89): a single-thread Gauss-Seidel sweep
// over every vertex with the same four functions until nothing changes
// (the host graph's V becomes that fixed point), then a comparison with the
// device values.  Prints PASSED or the first mismatch, as the reference does.
#ifndef KITES_B200_SANITY_CHECK_CUH_
#define KITES_B200_SANITY_CHECK_CUH_

#include <cstdio>
#include <cstdlib>
#include <iostream>

#include "graph_csr.h"
#include "graph_csr_device.cuh"
#include "graph_csr_mipmapped_device.cuh"

namespace kites {

template <class vT, class eT, class vIdxT, class FInit, class FComp, class FRed, class FUpd>
bool sanity_check(std::size_t n, host_pinned_buffer<vT> &V, host_pinned_buffer<vIdxT> &R,
                  host_pinned_buffer<vIdxT> &C, host_pinned_buffer<eT> &E, uva_buffer<vT> &devV,
                  FInit fInit, FComp fComp, FRed fRed, FUpd fUpd) {
  std::cout << "### SANITY CHECK ...\n";
  unsigned sweeps = 0;
  bool any;
  do {
    any = false;
    for (std::size_t v = 0; v < n; ++v) {
      vT pre = V[v];
      vT acc;
      fInit(acc, pre);
      for (std::size_t e = R[v]; e < R[v + 1]; ++e) {
        vT tmp;
        fComp(tmp, V.at(C.at(e)), E.get_ptr() + e);
        fRed(acc, tmp);
      }
      if (fUpd(acc, pre)) {
        V[v] = acc;
        any = true;
      }
    }
    ++sweeps;
  } while (any);
  std::cout << "### SANITY CHECK: Single CPU thread performed " << sweeps
            << " iterations in total.\n";
  host_pinned_buffer<vT> got(devV);
  // Test harnesses that run an unmodified program name a file in
  // KITES_SANITY_DUMP to receive the device values compared below (raw,
  // one vT per vertex).
  if (const char *dump = std::getenv("KITES_SANITY_DUMP")) {
    if (std::FILE *f = std::fopen(dump, "wb")) {
      std::fwrite(got.get_ptr(), sizeof(vT), got.size(), f);
      std::fclose(f);
    }
  }
  for (std::size_t i = 0; i < got.size(); ++i)
    if (!(got[i] == V[i])) {
      std::cout << "### SANITY CHECK: MISMATCH at index " << i << "! Expected " << V[i]
                << "\tbut got " << got[i] << "\n";
      return false;
    }
  std::cout << "### SANITY CHECK: PASSED!\n";
  return true;
}

template <class vT, class eT, class vIdxT, class FInit, class FComp, class FRed, class FUpd>
bool sanity_check(graph_csr<vT, eT, vIdxT> &h, graph_csr_device<vT, eT, vIdxT> &d, FInit fInit,
                  FComp fComp, FRed fRed, FUpd fUpd) {
  return sanity_check(h.get_num_vertices(), h.V, h.R, h.C, h.E, d.V, fInit, fComp, fRed, fUpd);
}

// kites/graph/sanity_check.cuh:82-89
template <class vT, class eT, class vIdxT, class FInit, class FComp, class FRed, class FUpd>
bool sanity_check(graph_csr_mipmapped<vT, eT, vIdxT> &h, graph_csr_mipmapped_device<vT, eT, vIdxT> &d,
                  FInit fInit, FComp fComp, FRed fRed, FUpd fUpd) {
  return sanity_check(h.get_num_vertices(), h.V, h.R, h.C, h.E, d.V, fInit, fComp, fRed, fUpd);
}

}  // namespace kites

#endif
