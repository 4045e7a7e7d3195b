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

/* ==========================================================================
 * Benchmark input graphs, restated independently of the product's
 * generator so that the reference arm of the benchmark can build its input
 * without loading the product library.  The rule (what is generated, not how):
 *   draw(base, i, j) = SplitMix64 finaliser of base + (64 i + j + 1) * golden
 *                      gamma (Steele, Lea, Flood, OOPSLA 2014), base =
 *                      finaliser(seed);
 *   R-MAT candidate i: for level l = 0..scale-1, r = draw(base, i, l) >> 32;
 *                      source bit = r >= a+b, destination bit =
 *                      (a <= r < a+b) or r >= a+b+c (thresholds are
 *                      floor(p * 2^32)); most significant level first;
 *   kept edges:        valid candidates (no self-loop, both ends < n) that
 *                      are the first occurrence of their (source, dest)
 *                      pair, in candidate order, the first n_edges of them;
 *   weight of the edge from candidate i: lo + ((draw(base, i, 63) >> 32) *
 *                      (hi - lo + 1)) >> 32.
 * First occurrences are found with a concurrent hash table (a minimum of
 * candidate index per pair), where the product sorts; both give the same
 * list, which tests/test_oracle.py checks.
 * ========================================================================== */
#include <stdlib.h>

static inline uint64_t kor_mix(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline uint64_t kor_draw(uint64_t base, uint64_t i, uint32_t j)
{
    return kor_mix(base + (i * 64ull + j + 1ull) * 0x9E3779B97F4A7C15ull);
}

static inline uint32_t kor_threshold(double p)
{
    double x = floor(p * 4294967296.0);
    return x >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)x;
}

typedef struct {
    uint32_t scale, t_a, t_ab, t_abc;
    uint64_t n, base;
} kor_rmat;

/* Candidate i of the R-MAT stream; returns 1 if it is a valid edge. */
static inline int kor_rmat_candidate(const kor_rmat *g, uint64_t i, uint32_t *s, uint32_t *d)
{
    uint32_t a = 0, b = 0;
    for (uint32_t l = 0; l < g->scale; ++l) {
        uint32_t r = (uint32_t)(kor_draw(g->base, i, l) >> 32);
        a = (a << 1) | (r >= g->t_ab ? 1u : 0u);
        b = (b << 1) | (((r >= g->t_a && r < g->t_ab) || r >= g->t_abc) ? 1u : 0u);
    }
    *s = a;
    *d = b;
    return a != b && a < g->n && b < g->n;
}

#define KOR_EMPTY 0xFFFFFFFFFFFFFFFFull

/* Slot of `key` in the open-addressing table (linear probing), inserting it
 * if absent. */
static uint64_t kor_slot(uint64_t *keys, uint64_t mask, uint64_t key)
{
    uint64_t h = kor_mix(key) & mask;
    for (;;) {
        uint64_t k = __atomic_load_n(&keys[h], __ATOMIC_RELAXED);
        if (k == key)
            return h;
        if (k == KOR_EMPTY) {
            uint64_t expected = KOR_EMPTY;
            if (__atomic_compare_exchange_n(&keys[h], &expected, key, 0, __ATOMIC_RELAXED,
                                            __ATOMIC_RELAXED) || expected == key)
                return h;
        }
        h = (h + 1) & mask;
    }
}

static void kor_atomic_min(uint64_t *p, uint64_t v)
{
    uint64_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
    while (v < cur && !__atomic_compare_exchange_n(p, &cur, v, 0, __ATOMIC_RELAXED,
                                                   __ATOMIC_RELAXED))
        ;
}

/* Read-only lookup of a key known to be in the table. */
static uint64_t kor_find(const uint64_t *keys, uint64_t mask, uint64_t key)
{
    uint64_t h = kor_mix(key) & mask;
    while (keys[h] != key)
        h = (h + 1) & mask;
    return h;
}

/* R-MAT edge list (see the rule above).  Returns 0, or -1 when memory runs
 * out or the stream cannot supply n_edges distinct edges. */
int kor_gen_rmat(uint32_t scale, uint64_t n_vertices, uint64_t n_edges, double a, double b,
                 double c, uint64_t seed, uint32_t w_lo, uint32_t w_hi, uint32_t *src,
                 uint32_t *dst, uint32_t *w)
{
    kor_rmat g;
    g.scale = scale;
    g.n = n_vertices ? n_vertices : (1ull << scale);
    g.t_a = kor_threshold(a);
    g.t_ab = kor_threshold(a + b);
    g.t_abc = kor_threshold(a + b + c);
    g.base = kor_mix(seed);
    uint64_t N = n_edges + n_edges / 4 + 4096;
    for (int attempt = 0; attempt < 12; ++attempt, N *= 2) {
        uint64_t T = 1024;
        while (T < N + N / 2)
            T <<= 1;
        uint64_t *cand = malloc(N * sizeof(uint64_t));   /* (s << 32 | d) or empty */
        uint64_t *keys = malloc(T * sizeof(uint64_t));
        uint64_t *first = malloc(T * sizeof(uint64_t));
        if (!cand || !keys || !first) {
            free(cand); free(keys); free(first);
            return -1;
        }
        memset(keys, 0xFF, T * sizeof(uint64_t));
        memset(first, 0xFF, T * sizeof(uint64_t));
        #pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
            uint32_t s, d;
            uint64_t key = KOR_EMPTY;
            if (kor_rmat_candidate(&g, (uint64_t)ii, &s, &d)) {
                key = (uint64_t)s << 32 | d;
                kor_atomic_min(&first[kor_slot(keys, T - 1, key)], (uint64_t)ii);
            }
            cand[ii] = key;
        }
        /* cand[i] keeps its key only for the first occurrence of the pair. */
        uint64_t kept = 0;
        #pragma omp parallel for schedule(static) reduction(+ : kept)
        for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
            if (cand[ii] == KOR_EMPTY)
                continue;
            if (first[kor_find(keys, T - 1, cand[ii])] == (uint64_t)ii)
                ++kept;
            else
                cand[ii] = KOR_EMPTY;
        }
        free(keys);
        free(first);
        if (kept < n_edges) {
            free(cand);
            continue;
        }
        /* Ordered compaction: per-block counts, their prefix, then writes. */
        const int64_t nb = 4096;
        uint64_t *boff = calloc(nb + 1, sizeof(uint64_t));
        if (!boff) {
            free(cand);
            return -1;
        }
        #pragma omp parallel for schedule(static)
        for (int64_t bi = 0; bi < nb; ++bi) {
            uint64_t lo = N * bi / nb, hi = N * (bi + 1) / nb, k = 0;
            for (uint64_t i = lo; i < hi; ++i)
                k += cand[i] != KOR_EMPTY;
            boff[bi + 1] = k;
        }
        for (int64_t bi = 0; bi < nb; ++bi)
            boff[bi + 1] += boff[bi];
        #pragma omp parallel for schedule(static)
        for (int64_t bi = 0; bi < nb; ++bi) {
            uint64_t o = boff[bi];
            for (uint64_t i = N * bi / nb; i < N * (bi + 1) / nb && o < n_edges; ++i) {
                if (cand[i] == KOR_EMPTY)
                    continue;
                src[o] = (uint32_t)(cand[i] >> 32);
                dst[o] = (uint32_t)cand[i];
                if (w) {
                    uint64_t r = kor_draw(g.base, i, 63) >> 32;
                    w[o] = w_lo + (uint32_t)((r * ((uint64_t)w_hi - w_lo + 1ull)) >> 32);
                }
                ++o;
            }
        }
        free(boff);
        free(cand);
        return 0;
    }
    return -1;
}

static int kor_cmp_u64(const void *x, const void *y)
{
    uint64_t a = *(const uint64_t *)x, b = *(const uint64_t *)y;
    return a < b ? -1 : (a > b);
}

/* CSC of an edge list: rows = destinations (R has n_vertices + 1 uint64
 * offsets), each row's sources ascending, edges with equal endpoints in
 * input order (graph_raw.h:102,131).  Each edge is placed in its row, then
 * the row is sorted by (source, input index).  Returns 0, or -1 on a bad
 * endpoint or when memory runs out. */
int kor_csc_from_edges(uint64_t n_vertices, uint64_t n_edges, const uint32_t *src,
                       const uint32_t *dst, const uint32_t *w, uint64_t *R, uint32_t *C,
                       uint32_t *E)
{
    if (n_edges > 0xFFFFFFFFull)
        return -1;
    uint64_t *cursor = calloc(n_vertices + 1, sizeof(uint64_t));
    uint64_t *slot = malloc((n_edges ? n_edges : 1) * sizeof(uint64_t));
    if (!cursor || !slot) {
        free(cursor); free(slot);
        return -1;
    }
    int bad = 0;
    #pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t i = 0; i < (int64_t)n_edges; ++i) {
        if (src[i] >= n_vertices || dst[i] >= n_vertices) {
            bad = 1;
            continue;
        }
        __atomic_fetch_add(&cursor[dst[i] + 1], 1ull, __ATOMIC_RELAXED);
    }
    if (bad) {
        free(cursor); free(slot);
        return -1;
    }
    R[0] = 0;
    for (uint64_t v = 0; v < n_vertices; ++v)
        R[v + 1] = R[v] + cursor[v + 1];
    memcpy(cursor, R, n_vertices * sizeof(uint64_t));
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n_edges; ++i) {
        uint64_t p = __atomic_fetch_add(&cursor[dst[i]], 1ull, __ATOMIC_RELAXED);
        slot[p] = (uint64_t)src[i] << 32 | (uint64_t)i;
    }
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t vi = 0; vi < (int64_t)n_vertices; ++vi) {
        uint64_t lo = R[vi], hi = R[vi + 1];
        if (hi - lo > 1)
            qsort(slot + lo, hi - lo, sizeof(uint64_t), kor_cmp_u64);
        for (uint64_t e = lo; e < hi; ++e) {
            C[e] = (uint32_t)(slot[e] >> 32);
            if (E)
                E[e] = w ? w[(uint32_t)slot[e]] : 0u;
        }
    }
    free(cursor);
    free(slot);
    return 0;
}

/*
 * Exact min-label connected components of the undirected graph behind an
 * edge list (each edge taken in both directions): union-find whose root is
 * always the smallest id of its set, so label[v] = the smallest vertex id in
 * v's component -- the fixed point of the min-label vertex program (init
 * V[v] = v, nbrComp = copy, reduce = min) on the symmetrised graph, reached
 * here without iterating.
 */
static uint32_t kor_root(uint32_t *parent, uint32_t x)
{
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];   /* path halving */
        x = parent[x];
    }
    return x;
}

void kor_cc_union_find(uint64_t n_vertices, uint64_t n_edges, const uint32_t *src,
                       const uint32_t *dst, uint32_t *label)
{
    for (uint64_t v = 0; v < n_vertices; ++v)
        label[v] = (uint32_t)v;
    for (uint64_t e = 0; e < n_edges; ++e) {
        uint32_t a = kor_root(label, src[e]), b = kor_root(label, dst[e]);
        if (a < b)
            label[b] = a;
        else if (b < a)
            label[a] = b;
    }
    for (uint64_t v = 0; v < n_vertices; ++v)
        label[v] = kor_root(label, (uint32_t)v);
}
