// kernels_mip.cuh -- the block map of kites::graph_csr_mipmapped
// (kites/graph/graph_csr_mipmapped.hpp:58-75, graph_csr_mipmapped_device.cuh:29-33)
// as an engine strategy: coarse activation over blocks of consecutive
// vertices.
//
// Layout, kept bit for bit from the reference class: blocks of `block`
// vertices, dim = ceil(n / block) rounded up to a multiple of 32, and a
// dim x dim row-major bit matrix with bit (s / block) * dim + d / block set
// for every edge s -> d (row = source block, one 32-bit word holds 32
// destination blocks).  n is the vertex count padded to a multiple of 128,
// as graph_raw pads it (graph_raw.h:174-179) and as the engine holds it.
//
// One MIP iteration: the changed vertex set U becomes a changed-block set
// (k_mip_blocks); the rows of the changed blocks are OR-ed into the set of
// active destination blocks (k_mip_activate, one coalesced pass over those
// rows); every vertex of an active block enters the read frontier
// (k_mip_expand); the frontier pull then runs as usual.  The frontier is a
// superset of the exact activation (every out-neighbour d of a changed s
// lies in a block that s's block has an edge into), so the fixed point is
// the same; the activation costs (changed blocks) x dim / 8 bytes instead
// of a walk over the changed vertices' out-edges.
#pragma once
#include "kernels.cuh"

namespace kites_internal {

// dim x dim bits stay under 2^32 (512 MiB), the reference's unsigned bit
// count (graph_csr_mipmapped.hpp:58-62).
constexpr uint64_t kMaxMipDim = 65536;

struct mip_geom {
  uint32_t *map;          // dim x dim bits
  uint64_t dim;           // blocks, a multiple of 32
  uint64_t row_words;     // dim / 32: words per map row and per block bitmap
  uint64_t block;         // vertices per block (>= 1)
};

// One warp per CSC row d (destination): every in-edge's source block s /
// block sets bit d / block of its map row.  Sources of a row ascend, so a
// lane's consecutive edges usually hit the same word; a word that already
// holds the bit costs a read and no atomic.
template <typename OffT>
__global__ void __launch_bounds__(256) k_mip_build(const OffT *R, const uint32_t *C,
                                                   uint64_t n_rows, mip_geom mg) {
  const uint32_t lane = lane_id();
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t d = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; d < n_rows;
       d += nwarps) {
    const uint64_t lo = (uint64_t)R[d], hi = (uint64_t)R[d + 1];
    const uint64_t col = d / mg.block;
    const uint32_t bit = 1u << (uint32_t)(col & 31u);
    uint64_t last = ~0ull;
    for (uint64_t j = lo + lane; j < hi; j += 32) {
      const uint64_t sb = (uint64_t)__ldg(C + j) / mg.block;
      if (sb >= mg.dim) continue;   // never: sources are real vertices
      const uint64_t w = sb * mg.row_words + (col >> 5);
      if (w == last) continue;
      last = w;
      if (!(mg.map[w] & bit)) atomicOr(mg.map + w, bit);
    }
  }
}

// Changed vertices -> changed blocks (bchg, dim bits); also clears the
// active-block set (bact) that the previous MIP iteration left.
__global__ void __launch_bounds__(256) k_mip_blocks(const uint32_t *U, uint64_t nwords,
                                                    mip_geom mg, uint32_t *bchg,
                                                    uint32_t *bact) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t top = max(nwords, mg.row_words);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < top; i += stride) {
    if (i < mg.row_words) bact[i] = 0u;
    if (i >= nwords) continue;
    uint32_t u = U[i];
    const uint64_t v0 = i * 32;
    while (u) {
      const uint32_t b = (uint32_t)__ffs(u) - 1u;
      const uint64_t blk = (v0 + b) / mg.block;
      // Bits of this word that lie in block blk are consumed at once.
      const uint64_t end = (blk + 1) * mg.block - v0;   // first bit past the block
      u = end >= 32 ? 0u : (u & (kFull << (uint32_t)end));
      if (blk >= mg.dim) break;   // never: dim x block covers every vertex
      uint32_t *w = bchg + (blk >> 5);
      const uint32_t bit = 1u << (uint32_t)(blk & 31u);
      if (!(*w & bit)) atomicOr(w, bit);
    }
  }
}

// Active destination blocks: thread x of slice y ORs map word x of every
// changed block whose bchg word index is y modulo the slices, so a row is
// read once, coalesced, by consecutive threads.
__global__ void __launch_bounds__(256) k_mip_activate(mip_geom mg, const uint32_t *bchg,
                                                      uint32_t *bact) {
  const uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= mg.row_words) return;
  uint32_t acc = 0u;
  for (uint64_t bw = blockIdx.y; bw < mg.row_words; bw += gridDim.y) {
    uint32_t word = bchg[bw];
    while (word) {
      const uint32_t b = (uint32_t)__ffs(word) - 1u;
      word &= word - 1u;
      acc |= __ldg(mg.map + (bw * 32 + b) * mg.row_words + x);
    }
  }
  if (acc) atomicOr(bact + x, acc);
}

// Active blocks -> read frontier A (vertex bits of the n vertices; A is
// clear on entry and has nwords >= n / 32 words).  Also clears bchg for the
// next MIP iteration.
__global__ void __launch_bounds__(256) k_mip_expand(uint32_t *A, uint64_t nwords, uint64_t n,
                                                    mip_geom mg, const uint32_t *bact,
                                                    uint32_t *bchg) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t top = max(nwords, mg.row_words);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < top; i += stride) {
    if (i < mg.row_words) bchg[i] = 0u;
    if (i >= nwords || i * 32 >= n) continue;   // n is a multiple of 32
    const uint64_t v0 = i * 32;
    uint32_t bits = 0u;
    for (uint64_t blk = v0 / mg.block; blk * mg.block < v0 + 32 && blk < mg.dim; ++blk) {
      if (!((bact[blk >> 5] >> (uint32_t)(blk & 31u)) & 1u)) continue;
      const uint64_t b0 = blk * mg.block > v0 ? blk * mg.block - v0 : 0;
      const uint64_t b1 = min((blk + 1) * mg.block - v0, (uint64_t)32);
      const uint32_t hi = b1 >= 32 ? kFull : ((1u << (uint32_t)b1) - 1u);
      bits |= hi & (kFull << (uint32_t)b0);
    }
    if (bits) A[i] = bits;
  }
}

}  // namespace kites_internal
