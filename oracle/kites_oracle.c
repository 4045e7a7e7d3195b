/*
 * kites_oracle.c -- CPU restatement of farkhor/KiTES's single-GPU
 * vertex-centric path, used ONLY as the checker by tests/, by
 * __graft_entry__.smoke() and by bench.py's cpu_baseline leg.  Nothing in
 * the product (kites_b200/, include/) links, loads or calls this file.
 *
 * What is restated (reference paths relative to the KiTES project root):
 *   kor_sanity_check   kites/graph/sanity_check.cuh:13-59  -- the single-thread
 *                      Gauss-Seidel sweep over all vertices until no update.
 *   kor_process        kites/device/compute.cuh:29-137 driving
 *                      kites/device/kernels_single_device.cuh:18-426 -- the
 *                      frontier-driven iteration (bitmap ping-pong, in-place
 *                      vertex updates, out-neighbour activation, vpg groups),
 *                      executed sequentially (one valid schedule of the
 *                      asynchronous in-place kernel).
 *   kor_pagerank_f64   FP64 Jacobi PageRank used as the tolerance oracle for
 *                      FP32 PageRank (the reference has no PR; the rule is
 *                      PR <- (1-d)/n + d * sum_{u->v} PR(u)/outdeg(u), uniform
 *                      1/n start, no dangling redistribution).
 *
 * The operators are the four user functions of the reference's SSSP example
 * (examples/sssp_basic_single_device.cu:40-47) and their BFS / CC variants:
 *   KOR_SSSP_WRAP  partial = src + w            (u32 wrap-around, as written in
 *                                                the example's lambda)
 *   KOR_SSSP_SAT   partial = src + w, saturating at 0xFFFFFFFF
 *   KOR_BFS_SAT    partial = src + 1, saturating
 *   KOR_CC_MIN     partial = src                 (min-label)
 * each with init = copy, reduce = min, update = (new < old).
 *
 * Edge offsets are taken as uint64 here; the reference stores them as
 * uint32 and masks bit 31 (sanity_check.cuh:25), which is a no-op for the
 * graph sizes the oracle runs on.
 */
#include <stdint.h>
#include <stddef.h>
#include <string.h>
#include <math.h>

enum {
    KOR_SSSP_WRAP = 0,
    KOR_SSSP_SAT = 1,
    KOR_BFS_SAT = 2,
    KOR_CC_MIN = 3
};

static inline uint32_t kor_comp(int op, uint32_t src, uint32_t w)
{
    uint32_t s;
    switch (op) {
    case KOR_SSSP_WRAP:
        return src + w;
    case KOR_SSSP_SAT:
        s = src + w;
        return (s < src) ? 0xFFFFFFFFu : s;
    case KOR_BFS_SAT:
        return (src == 0xFFFFFFFFu) ? 0xFFFFFFFFu : src + 1u;
    default: /* KOR_CC_MIN */
        return src;
    }
}

/*
 * sanity_check.cuh:22-47.  V is updated in place to the fixed point;
 * returns the number of sweeps (the reference's iterationCounter, which
 * counts the final no-update sweep too).
 */
uint64_t kor_sanity_check(int op, uint64_t n_vertices, const uint64_t *R,
                          const uint32_t *C, const uint32_t *E, uint32_t *V)
{
    uint64_t sweeps = 0;
    int any;
    do {
        any = 0;
        for (uint64_t v = 0; v < n_vertices; ++v) {
            uint32_t pre = V[v];
            uint32_t acc = pre;                       /* initF: copy        */
            for (uint64_t e = R[v]; e < R[v + 1]; ++e) {
                uint32_t t = kor_comp(op, V[C[e]], E ? E[e] : 1u);
                if (acc > t)                          /* redF: min          */
                    acc = t;
            }
            if (acc < pre) {                          /* updF: new < old    */
                V[v] = acc;
                any = 1;
            }
        }
        ++sweeps;
    } while (any);
    return sweeps;
}

static inline int kor_bit(const uint32_t *bits, uint64_t nbits, uint64_t i)
{
    /* The reference reads bits past the allocated bitmap for the padded
     * tail when vpg > 1 (graph_raw.h:93 vs :173-182); treat them as 0. */
    if (i >= nbits)
        return 0;
    return (bits[i >> 5] >> (i & 31)) & 1u;
}

static inline void kor_set(uint32_t *bits, uint64_t nbits, uint64_t i)
{
    if (i < nbits)
        bits[i >> 5] |= 1u << (i & 31);
}

/*
 * compute.cuh:57-128 with kernels_single_device.cuh.  The two bitmaps have
 * nbits bits each (words = ceil(nbits/32)); even_bits holds the initial
 * frontier on entry.  For vpg == 1 a bit is a vertex; for vpg > 1 a bit is
 * a group of vpg consecutive vertices and the activation adjacency dir_R /
 * dir_C is group-level.  directed == 0 activates through C (the symmetric
 * in-neighbour list, kernels_single_device.cuh:161-163).
 * Returns the number of iterations (kernel launches) performed.
 */
uint64_t kor_process(int op, uint64_t n_vertices, const uint64_t *R,
                     const uint32_t *C, const uint32_t *E, uint32_t *V,
                     uint32_t vpg, int directed, const uint64_t *dir_R,
                     const uint32_t *dir_C, uint32_t *even_bits,
                     uint32_t *odd_bits, uint64_t nbits, uint32_t *updated_scratch,
                     uint64_t max_iterations)
{
    uint64_t iters = 0;
    uint64_t nwords = (nbits + 31) / 32;
    uint32_t shift = 0;
    while ((1u << shift) < vpg)
        ++shift;
    int any;
    do {
        uint32_t *rd = (iters & 1) ? odd_bits : even_bits;
        uint32_t *wr = (iters & 1) ? even_bits : odd_bits;
        any = 0;
        /* updated_scratch: one flag per group (vpg > 1) or per vertex. */
        uint64_t ngroups = (n_vertices + vpg - 1) / vpg;
        memset(updated_scratch, 0, ngroups * sizeof(uint32_t));
        for (uint64_t v = 0; v < n_vertices; ++v) {
            uint64_t g = v >> shift;
            if (!kor_bit(rd, nbits, g))
                continue;
            uint32_t old = V[v];
            uint32_t acc = old;
            for (uint64_t e = R[v]; e < R[v + 1]; ++e) {
                uint32_t t = kor_comp(op, V[C[e]], E ? E[e] : 1u);
                if (acc > t)
                    acc = t;
            }
            if (acc < old) {
                V[v] = acc;
                any = 1;
                if (vpg == 1) {
                    if (directed) {
                        for (uint64_t j = dir_R[v]; j < dir_R[v + 1]; ++j)
                            kor_set(wr, nbits, dir_C[j]);
                    } else {
                        for (uint64_t e = R[v]; e < R[v + 1]; ++e)
                            kor_set(wr, nbits, C[e]);
                    }
                } else {
                    updated_scratch[g] = 1;
                }
            }
        }
        if (vpg != 1) {
            for (uint64_t g = 0; g < ngroups; ++g)
                if (updated_scratch[g])
                    for (uint64_t j = dir_R[g]; j < dir_R[g + 1]; ++j)
                        kor_set(wr, nbits, dir_C[j]);
        }
        memset(rd, 0, nwords * sizeof(uint32_t));  /* compute.cuh:121 */
        ++iters;
    } while (any && iters < max_iterations);
    return iters;
}

/*
 * FP64 Jacobi PageRank over the CSC (rows = destinations).  out_degree[u]
 * is the number of out-edges of u; vertices >= n_real (padding) keep 0.
 */
void kor_pagerank_f64(uint64_t n_real, const uint64_t *R, const uint32_t *C,
                      const uint32_t *out_degree, uint32_t iterations,
                      double damping, double *pr, double *tmp)
{
    double base = (1.0 - damping) / (double)n_real;
    for (uint64_t v = 0; v < n_real; ++v)
        pr[v] = 1.0 / (double)n_real;
    for (uint32_t it = 0; it < iterations; ++it) {
        /* Rows are independent within a Jacobi step and each row sums its
         * in-edges in CSC order, so the threads change no result. */
        #pragma omp parallel for schedule(dynamic, 4096)
        for (int64_t vi = 0; vi < (int64_t)n_real; ++vi) {
            const uint64_t v = (uint64_t)vi;
            double s = 0.0;
            for (uint64_t e = R[v]; e < R[v + 1]; ++e) {
                uint32_t u = C[e];
                s += pr[u] / (double)out_degree[u];
            }
            tmp[v] = base + damping * s;
        }
        memcpy(pr, tmp, n_real * sizeof(double));
    }
}

/*
 * Plain Bellman-Ford/BFS/CC by label-correcting queue, independent of the
 * sweep order above; used in tests to cross-check kor_sanity_check on
 * random inputs (both must reach the same unique fixed point).
 */
uint64_t kor_jacobi_fixed_point(int op, uint64_t n_vertices, const uint64_t *R,
                                const uint32_t *C, const uint32_t *E,
                                uint32_t *V, uint32_t *next)
{
    uint64_t rounds = 0;
    int any;
    do {
        any = 0;
        for (uint64_t v = 0; v < n_vertices; ++v) {
            uint32_t acc = V[v];
            for (uint64_t e = R[v]; e < R[v + 1]; ++e) {
                uint32_t t = kor_comp(op, V[C[e]], E ? E[e] : 1u);
                if (acc > t)
                    acc = t;
            }
            next[v] = acc;
            if (acc < V[v])
                any = 1;
        }
        memcpy(V, next, n_vertices * sizeof(uint32_t));
        ++rounds;
    } while (any);
    return rounds;
}
