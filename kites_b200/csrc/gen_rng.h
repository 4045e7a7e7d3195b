// gen_rng.h -- counter-based synthetic-graph draws shared by the host
// generators (host/graphgen.cpp) and any device generator.
//
// Every draw is one output of SplitMix64 (Steele, Lea, Flood, "Fast
// splittable pseudorandom number generators", OOPSLA 2014): the state is a
// Weyl sequence base + k * 0x9E3779B97F4A7C15 and each output is the
// published MurmurHash3-style finaliser of the state.  Candidate edge i uses
// stream positions k = 64 i + j + 1 (j = level 0..scale-1 for the R-MAT
// quadrant draws, j = 0/1 for ER endpoints, j = 63 for the weight), so any
// edge can be generated independently of the others, in any order, on any
// device.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define KITES_HD __host__ __device__ __forceinline__
#else
#define KITES_HD inline
#endif

namespace kites_gen {

KITES_HD uint64_t splitmix64_finalise(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

KITES_HD uint64_t draw(uint64_t base, uint64_t edge, uint32_t j) {
  return splitmix64_finalise(base + (edge * 64ull + j + 1ull) *
                                        0x9E3779B97F4A7C15ull);
}

KITES_HD uint64_t stream_base(uint64_t seed) {
  return splitmix64_finalise(seed);
}

// Uniform in [lo, hi] from the high 32 bits (multiply-high, no modulo).
KITES_HD uint32_t uniform_u32(uint64_t r, uint32_t lo, uint32_t hi) {
  uint64_t range = (uint64_t)hi - lo + 1ull;
  return lo + (uint32_t)(((r >> 32) * range) >> 32);
}

// Uniform in [0, n) for n <= 2^32.
KITES_HD uint32_t uniform_below(uint64_t r, uint64_t n) {
  return (uint32_t)(((r >> 32) * n) >> 32);
}

struct rmat_thresholds {
  uint32_t a, ab, abc;
};

// R-MAT quadrant choice per level: r < a -> (0,0); < a+b -> (0,1);
// < a+b+c -> (1,0); else (1,1); row bit = source, column bit = destination.
KITES_HD void rmat_edge(uint64_t base, uint64_t edge, uint32_t scale,
                        rmat_thresholds t, uint32_t *src, uint32_t *dst) {
  uint32_t s = 0, d = 0;
  for (uint32_t l = 0; l < scale; ++l) {
    uint32_t r = (uint32_t)(draw(base, edge, l) >> 32);
    uint32_t sb = (r >= t.ab) ? 1u : 0u;
    uint32_t db = (r >= t.a && r < t.ab) || (r >= t.abc) ? 1u : 0u;
    s = (s << 1) | sb;
    d = (d << 1) | db;
  }
  *src = s;
  *dst = d;
}

}  // namespace kites_gen
