// graphgen.cpp -- deterministic synthetic graphs and the host edge-list ->
// CSC builder (OpenMP).  Input creation for tests, benchmarks and selector
// training; the CSC layout follows kites/graph/graph_raw.h:102,131 (rows are
// destinations, each row sorted by source, ties kept in input order).
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "../gen_rng.h"
#include "kites_b200.h"
#include "../status.h"

namespace {

struct rec {
  uint64_t key;
  uint32_t val;
  uint32_t pad;
};

// Parallel LSD radix sort of records by the low `bits` bits of key; stable.
void radix_sort(std::vector<rec> &a, uint32_t bits) {
  const int kDigit = 11;
  const size_t kBuckets = size_t(1) << kDigit;
  const size_t n = a.size();
  if (n < 2 || bits == 0) return;
  std::vector<rec> b(n);
  // Partition by the size of the team actually running (1 when called from
  // inside another parallel region).
  const int max_threads = omp_get_max_threads();
  std::vector<size_t> hist(kBuckets * max_threads);
  rec *src = a.data(), *dst = b.data();
  int passes = 0;
  for (uint32_t shift = 0; shift < bits; shift += kDigit, ++passes) {
    std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(max_threads)
    {
      const int nthreads = omp_get_num_threads();
      int t = omp_get_thread_num();
      size_t lo = n * t / nthreads, hi = n * (t + 1) / nthreads;
      size_t *h = &hist[kBuckets * t];
      for (size_t i = lo; i < hi; ++i) ++h[(src[i].key >> shift) & (kBuckets - 1)];
#pragma omp barrier
#pragma omp single
      {
        size_t run = 0;
        for (size_t d = 0; d < kBuckets; ++d)
          for (int tt = 0; tt < nthreads; ++tt) {
            size_t c = hist[kBuckets * tt + d];
            hist[kBuckets * tt + d] = run;
            run += c;
          }
      }
      for (size_t i = lo; i < hi; ++i) {
        size_t d = (src[i].key >> shift) & (kBuckets - 1);
        dst[h[d]++] = src[i];
      }
    }
    std::swap(src, dst);
  }
  if (src != a.data()) a.swap(b);
}

template <class CandFn>
int dedup_topup(uint64_t n_edges, uint32_t key_bits, CandFn cand,
                uint32_t *src, uint32_t *dst, uint32_t *w) {
  uint64_t N = n_edges + n_edges / 8 + 1024;
  for (int attempt = 0; attempt < 40; ++attempt) {
    std::vector<rec> r;
    std::vector<uint8_t> keep;
    try {
      r.resize(N);
      keep.assign(N, 0);
    } catch (const std::bad_alloc &) {
      return kites_internal::fail(KITES_ERR_OOM, "host allocation of %llu candidates failed",
                                  (unsigned long long)N);
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)N; ++i) {
      uint32_t s, d;
      bool ok = cand((uint64_t)i, &s, &d);
      // Invalid candidates get a key above every valid one.
      r[i].key = ok ? ((uint64_t)s << 32 | d) : ~0ull;
      r[i].val = (uint32_t)i;
      r[i].pad = ok ? 1u : 0u;
    }
    if (N > 0xFFFFFFFFull)
      return kites_internal::fail(KITES_ERR_INVALID, "too many candidates");
    // Sort by (src, dst) keeping candidate order among duplicates: the
    // first of each run is the first occurrence.  Keys use 64 bits so that
    // the invalid marker sorts last.
    (void)key_bits;
    radix_sort(r, 64);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)N; ++i) {
      if (!r[i].pad) continue;
      if (i == 0 || r[i - 1].key != r[i].key) keep[r[i].val] = 1;
    }
    uint64_t kept = 0;
#pragma omp parallel for reduction(+ : kept) schedule(static)
    for (int64_t i = 0; i < (int64_t)N; ++i) kept += keep[i];
    if (kept < n_edges) {
      double f = kept ? (double)n_edges / (double)kept : 2.0;
      N = (uint64_t)(N * std::min(4.0, f * 1.15)) + 4096;
      continue;
    }
    // Ordered compaction of the first n_edges kept candidates.
    const int max_threads = omp_get_max_threads();
    std::vector<uint64_t> counts(max_threads + 1, 0);
#pragma omp parallel num_threads(max_threads)
    {
      const int nthreads = omp_get_num_threads();
      int t = omp_get_thread_num();
      uint64_t lo = N * t / nthreads, hi = N * (t + 1) / nthreads, c = 0;
      for (uint64_t i = lo; i < hi; ++i) c += keep[i];
      counts[t + 1] = c;
#pragma omp barrier
#pragma omp single
      for (int tt = 0; tt < nthreads; ++tt) counts[tt + 1] += counts[tt];
      uint64_t o = counts[t];
      for (uint64_t i = lo; i < hi && o < n_edges; ++i) {
        if (!keep[i]) continue;
        uint32_t s, d;
        cand(i, &s, &d);
        src[o] = s;
        dst[o] = d;
        if (w) w[o] = (uint32_t)i;  // candidate index, replaced by the caller
        ++o;
      }
    }
    return KITES_OK;
  }
  return kites_internal::fail(KITES_ERR_INVALID,
                              "could not reach %llu distinct edges",
                              (unsigned long long)n_edges);
}

}  // namespace

extern "C" int kites_gen_rmat(uint32_t scale, uint64_t n_vertices,
                              uint64_t n_edges, double a, double b, double c,
                              uint64_t seed, uint32_t w_lo, uint32_t w_hi,
                              uint32_t *src, uint32_t *dst, uint32_t *w) {
  kites_internal::clear_error();
  if (scale == 0 || scale > 31 || !src || !dst || w_lo > w_hi)
    return kites_internal::fail(KITES_ERR_INVALID, "bad R-MAT arguments");
  if (n_vertices == 0) n_vertices = 1ull << scale;
  if (n_vertices > (1ull << scale))
    return kites_internal::fail(KITES_ERR_INVALID, "n_vertices > 2^scale");
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
    return kites_internal::fail(KITES_ERR_INVALID, "bad R-MAT probabilities");
  auto thr = [](double p) -> uint32_t {
    double x = std::floor(p * 4294967296.0);
    return x >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)x;
  };
  kites_gen::rmat_thresholds t{thr(a), thr(a + b), thr(a + b + c)};
  const uint64_t base = kites_gen::stream_base(seed);
  auto cand = [&](uint64_t i, uint32_t *s, uint32_t *d) {
    kites_gen::rmat_edge(base, i, scale, t, s, d);
    return *s != *d && *s < n_vertices && *d < n_vertices;
  };
  int st = dedup_topup(n_edges, 2 * scale, cand, src, dst, w);
  if (st != KITES_OK || !w) return st;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n_edges; ++i)
    w[i] = kites_gen::uniform_u32(kites_gen::draw(base, w[i], 63), w_lo, w_hi);
  return KITES_OK;
}

extern "C" int kites_gen_er(uint64_t n_vertices, uint64_t n_edges,
                            uint64_t seed, uint32_t w_lo, uint32_t w_hi,
                            uint32_t *src, uint32_t *dst, uint32_t *w) {
  kites_internal::clear_error();
  if (n_vertices < 2 || n_vertices > 0xFFFFFFFFull || !src || !dst || w_lo > w_hi)
    return kites_internal::fail(KITES_ERR_INVALID, "bad ER arguments");
  if ((double)n_edges > 0.5 * (double)n_vertices * (double)(n_vertices - 1))
    return kites_internal::fail(KITES_ERR_INVALID, "ER graph too dense");
  const uint64_t base = kites_gen::stream_base(seed);
  auto cand = [&](uint64_t i, uint32_t *s, uint32_t *d) {
    *s = kites_gen::uniform_below(kites_gen::draw(base, i, 0), n_vertices);
    *d = kites_gen::uniform_below(kites_gen::draw(base, i, 1), n_vertices);
    return *s != *d;
  };
  int st = dedup_topup(n_edges, 64, cand, src, dst, w);
  if (st != KITES_OK || !w) return st;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n_edges; ++i)
    w[i] = kites_gen::uniform_u32(kites_gen::draw(base, w[i], 63), w_lo, w_hi);
  return KITES_OK;
}

extern "C" int kites_gen_grid(uint32_t side, uint64_t seed, uint32_t w_lo,
                              uint32_t w_hi, uint32_t *src, uint32_t *dst,
                              uint32_t *w) {
  kites_internal::clear_error();
  if (side < 2 || (uint64_t)side * side > 0xFFFFFFFFull || !src || !dst || w_lo > w_hi)
    return kites_internal::fail(KITES_ERR_INVALID, "bad grid arguments");
  const uint64_t base = kites_gen::stream_base(seed);
  // Per vertex in id order: right, down, left, up neighbours that exist.
  // Interior vertices have 4 edges; edge slots are counted per row.
  const uint64_t n = (uint64_t)side * side;
  std::vector<uint64_t> start(n + 1, 0);
  auto deg = [&](uint64_t v) {
    uint32_t r = (uint32_t)(v / side), c = (uint32_t)(v % side);
    return (uint64_t)((c + 1 < side) + (r + 1 < side) + (c > 0) + (r > 0));
  };
  for (uint64_t v = 0; v < n; ++v) start[v + 1] = start[v] + deg(v);
#pragma omp parallel for schedule(static)
  for (int64_t vi = 0; vi < (int64_t)n; ++vi) {
    uint64_t v = (uint64_t)vi, o = start[v];
    uint32_t r = (uint32_t)(v / side), c = (uint32_t)(v % side);
    uint64_t nb[4];
    int k = 0;
    if (c + 1 < side) nb[k++] = v + 1;
    if (r + 1 < side) nb[k++] = v + side;
    if (c > 0) nb[k++] = v - 1;
    if (r > 0) nb[k++] = v - side;
    for (int j = 0; j < k; ++j, ++o) {
      src[o] = (uint32_t)v;
      dst[o] = (uint32_t)nb[j];
      if (w) w[o] = kites_gen::uniform_u32(kites_gen::draw(base, o, 63), w_lo, w_hi);
    }
  }
  return KITES_OK;
}

extern "C" int kites_csc_from_edges(uint64_t n_vertices, uint64_t n_edges,
                                    const uint32_t *src, const uint32_t *dst,
                                    const uint32_t *w, uint64_t *R,
                                    uint32_t *C, uint32_t *E) {
  kites_internal::clear_error();
  if (!R || (n_edges && (!src || !dst || !C)))
    return kites_internal::fail(KITES_ERR_INVALID, "null CSC argument");
  std::vector<rec> r;
  try {
    r.resize(n_edges);
  } catch (const std::bad_alloc &) {
    return kites_internal::fail(KITES_ERR_OOM, "host allocation failed");
  }
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (int64_t i = 0; i < (int64_t)n_edges; ++i) {
    if (src[i] >= n_vertices || dst[i] >= n_vertices) bad = 1;
    r[i].key = (uint64_t)dst[i] << 32 | src[i];
    r[i].val = w ? w[i] : 0u;
  }
  if (bad) return kites_internal::fail(KITES_ERR_INVALID, "edge endpoint >= n_vertices");
  radix_sort(r, 64);
  memset(R, 0, (n_vertices + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < n_edges; ++i) ++R[(r[i].key >> 32) + 1];
  for (uint64_t v = 0; v < n_vertices; ++v) R[v + 1] += R[v];
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n_edges; ++i) {
    C[i] = (uint32_t)(r[i].key & 0xFFFFFFFFu);
    if (E) E[i] = r[i].val;
  }
  return KITES_OK;
}

// Disjoint union of n_graphs R-MAT graphs (a,b,c = 0.57,0.19,0.19): graph i
// has V_i log-uniform in [v_min, v_max] and edge factor uniform in
// [ef_min, ef_max] (one SplitMix64 stream per graph for the sizes, seed
// seed * 1000003 + i for its edges); vertex ids of graph i are shifted by
// vertex_offsets[i].  With src == NULL only the offsets are computed.
extern "C" int kites_gen_rmat_union(uint32_t n_graphs, uint64_t seed, uint32_t v_min,
                                    uint32_t v_max, uint32_t ef_min, uint32_t ef_max,
                                    uint32_t w_lo, uint32_t w_hi, uint64_t *vertex_offsets,
                                    uint64_t *edge_offsets, uint32_t *src, uint32_t *dst,
                                    uint32_t *w) {
  kites_internal::clear_error();
  if (!n_graphs || v_min < 2 || v_max < v_min || ef_max < ef_min || !ef_min ||
      !vertex_offsets || !edge_offsets || w_lo > w_hi)
    return kites_internal::fail(KITES_ERR_INVALID, "bad union arguments");
  const uint64_t base = kites_gen::stream_base(seed ^ 0x5eed5eedull);
  vertex_offsets[0] = edge_offsets[0] = 0;
  std::vector<uint32_t> nv(n_graphs), ef(n_graphs);
  for (uint32_t i = 0; i < n_graphs; ++i) {
    const double u = (double)(kites_gen::draw(base, i, 0) >> 11) * (1.0 / 9007199254740992.0);
    const double lv = std::log((double)v_min) + u * (std::log((double)v_max) - std::log((double)v_min));
    nv[i] = std::min<uint32_t>(v_max, std::max<uint32_t>(v_min, (uint32_t)std::floor(std::exp(lv))));
    ef[i] = kites_gen::uniform_u32(kites_gen::draw(base, i, 1), ef_min, ef_max);
    vertex_offsets[i + 1] = vertex_offsets[i] + nv[i];
    edge_offsets[i + 1] = edge_offsets[i] + (uint64_t)nv[i] * ef[i];
  }
  if (vertex_offsets[n_graphs] > 0xFFFFFF00ull)
    return kites_internal::fail(KITES_ERR_INVALID, "union exceeds 32-bit vertex ids");
  if (!src) return KITES_OK;
  if (!dst) return kites_internal::fail(KITES_ERR_INVALID, "null dst");
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
  for (int64_t i = 0; i < (int64_t)n_graphs; ++i) {
    uint32_t scale = 1;
    while ((1u << scale) < nv[i]) ++scale;
    const uint64_t eo = edge_offsets[i], m = edge_offsets[i + 1] - eo;
    if (kites_gen_rmat(scale, nv[i], m, 0.57, 0.19, 0.19, seed * 1000003ull + (uint64_t)i, w_lo,
                       w_hi, src + eo, dst + eo, w ? w + eo : nullptr) != KITES_OK) {
      bad = 1;
      continue;
    }
    const uint32_t vo = (uint32_t)vertex_offsets[i];
    for (uint64_t e = 0; e < m; ++e) {
      src[eo + e] += vo;
      dst[eo + e] += vo;
    }
  }
  if (bad) return kites_internal::fail(KITES_ERR_INVALID, "a union member could not be generated");
  return KITES_OK;
}

// ---- binary CSC files ------------------------------------------------------
//
// The prepared text format of the reference (kites/io/graph_output.cuh:23-38,
// read back by kites/graph/graph_csr.h:112-166) holds one value per line; at
// R-MAT scale 24 that is about 6 GB of text and minutes of parsing.  This is
// the same CSC as raw little-endian arrays behind a 128-byte header:
//   char     magic[8]      "KITESCSC"
//   uint32   version       1
//   uint32   flags         1: edge values present, 2: directed
//   uint64   n_vertices, n_edges
//   uint64   reserved      0
//   char     desc[88]      NUL-padded ASCII: how the graph was made
// then R (n_vertices + 1 uint64), C (n_edges uint32), E (n_edges uint32, if
// flag 1).  Files are written under a temporary name and renamed, so a
// reader never sees a partial file.
namespace {

struct csc_file_header {
  char magic[8];
  uint32_t version;
  uint32_t flags;
  uint64_t n_vertices;
  uint64_t n_edges;
  uint64_t reserved;
  char desc[88];
};
static_assert(sizeof(csc_file_header) == 128, "CSC file header is 128 bytes");

constexpr char kCscMagic[8] = {'K', 'I', 'T', 'E', 'S', 'C', 'S', 'C'};

bool write_all(FILE *f, const void *p, size_t bytes) {
  return bytes == 0 || fwrite(p, 1, bytes, f) == bytes;
}

bool read_all(FILE *f, void *p, size_t bytes) {
  return bytes == 0 || fread(p, 1, bytes, f) == bytes;
}

int read_csc_header(const char *path, FILE **fout, csc_file_header *h) {
  FILE *f = fopen(path, "rb");
  if (!f) return kites_internal::fail(KITES_ERR_INVALID, "cannot open %s", path);
  if (!read_all(f, h, sizeof(*h)) || memcmp(h->magic, kCscMagic, 8) != 0 || h->version != 1) {
    fclose(f);
    return kites_internal::fail(KITES_ERR_INVALID, "%s is not a version-1 CSC file", path);
  }
  const uint64_t want = sizeof(*h) + 8ull * (h->n_vertices + 1) +
                        4ull * h->n_edges * ((h->flags & 1u) ? 2u : 1u);
  if (fseeko(f, 0, SEEK_END) != 0 || (uint64_t)ftello(f) != want ||
      fseeko(f, sizeof(*h), SEEK_SET) != 0) {
    fclose(f);
    return kites_internal::fail(KITES_ERR_INVALID, "%s is truncated or has trailing bytes", path);
  }
  *fout = f;
  return KITES_OK;
}

}  // namespace

extern "C" int kites_csc_save(const char *path, uint64_t n_vertices, uint64_t n_edges,
                              const uint64_t *R, const uint32_t *C, const uint32_t *E,
                              int directed, const char *desc) {
  kites_internal::clear_error();
  if (!path || !R || (n_edges && !C))
    return kites_internal::fail(KITES_ERR_INVALID, "null CSC file argument");
  if (R[0] != 0 || R[n_vertices] != n_edges)
    return kites_internal::fail(KITES_ERR_INVALID, "R does not span 0 .. n_edges");
  csc_file_header h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, kCscMagic, 8);
  h.version = 1;
  h.flags = (E ? 1u : 0u) | (directed ? 2u : 0u);
  h.n_vertices = n_vertices;
  h.n_edges = n_edges;
  if (desc) strncpy(h.desc, desc, sizeof(h.desc) - 1);
  char tmp[4096];
  if (snprintf(tmp, sizeof(tmp), "%s.tmp%ld", path, (long)getpid()) >= (int)sizeof(tmp))
    return kites_internal::fail(KITES_ERR_INVALID, "path too long");
  FILE *f = fopen(tmp, "wb");
  if (!f) return kites_internal::fail(KITES_ERR_INVALID, "cannot create %s", tmp);
  bool ok = write_all(f, &h, sizeof(h)) && write_all(f, R, 8ull * (n_vertices + 1)) &&
            write_all(f, C, 4ull * n_edges) && (!E || write_all(f, E, 4ull * n_edges));
  ok = (fclose(f) == 0) && ok;
  if (!ok || rename(tmp, path) != 0) {
    remove(tmp);
    return kites_internal::fail(KITES_ERR_INVALID, "writing %s failed", path);
  }
  return KITES_OK;
}

extern "C" int kites_csc_info(const char *path, uint64_t *n_vertices, uint64_t *n_edges,
                              int *has_values, int *directed, char *desc, size_t desc_len) {
  kites_internal::clear_error();
  if (!path) return kites_internal::fail(KITES_ERR_INVALID, "null path");
  FILE *f = nullptr;
  csc_file_header h;
  int st = read_csc_header(path, &f, &h);
  if (st != KITES_OK) return st;
  fclose(f);
  if (n_vertices) *n_vertices = h.n_vertices;
  if (n_edges) *n_edges = h.n_edges;
  if (has_values) *has_values = (h.flags & 1u) ? 1 : 0;
  if (directed) *directed = (h.flags & 2u) ? 1 : 0;
  if (desc && desc_len) {
    const size_t k = std::min(desc_len - 1, strnlen(h.desc, sizeof(h.desc)));
    memcpy(desc, h.desc, k);
    desc[k] = '\0';
  }
  return KITES_OK;
}

extern "C" int kites_csc_load(const char *path, uint64_t *R, uint32_t *C, uint32_t *E) {
  kites_internal::clear_error();
  if (!path || !R) return kites_internal::fail(KITES_ERR_INVALID, "null CSC file argument");
  FILE *f = nullptr;
  csc_file_header h;
  int st = read_csc_header(path, &f, &h);
  if (st != KITES_OK) return st;
  if (h.n_edges && !C) {
    fclose(f);
    return kites_internal::fail(KITES_ERR_INVALID, "null C for a graph with edges");
  }
  bool ok = read_all(f, R, 8ull * (h.n_vertices + 1)) && read_all(f, C, 4ull * h.n_edges);
  if (ok && (h.flags & 1u)) {
    if (E) ok = read_all(f, E, 4ull * h.n_edges);
  }
  fclose(f);
  if (!ok) return kites_internal::fail(KITES_ERR_INVALID, "reading %s failed", path);
  if (R[0] != 0 || R[h.n_vertices] != h.n_edges)
    return kites_internal::fail(KITES_ERR_INVALID, "%s: R does not span 0 .. n_edges", path);
  return KITES_OK;
}
