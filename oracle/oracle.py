"""CPU oracle for the KiTES single-GPU ``process`` path -- TEST INFRASTRUCTURE.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s cpu_baseline
leg import this module, and only as the checker.  The product path
(``kites_b200`` and ``include/``) never imports it.

Contents
  build_host_graph   restates graph_raw.h:57-190 + graph_csr.h:44-110 (the
                     host CSC, initial values, initial frontier bitmap,
                     128-padding and the vpg group out-adjacency) in numpy.
  mipmap_of          the block frontier and block mipmap of
                     graph_csr_mipmapped.hpp:40-78.
  sanity_check       kites/graph/sanity_check.cuh:22-47 (C, kites_oracle.c)
  process            kites/device/compute.cuh:29-137 + kernels_single_device.cuh
                     restated sequentially (C, kites_oracle.c)
  pagerank_f64       FP64 Jacobi PageRank oracle (C)
  certify_*          size-independent fixed-point certificates used at sizes
                     the sequential oracle cannot finish in seconds.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libkites_oracle.so")

OP_SSSP_WRAP = 0
OP_SSSP_SAT = 1
OP_BFS_SAT = 2
OP_CC_MIN = 3

INF32 = 0xFFFFFFFF


def build_oracle_lib() -> str:
    """Compile kites_oracle.c with gcc into oracle/_build/ (idempotent)."""
    src = os.path.join(HERE, "kites_oracle.c")
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    if (not os.path.exists(LIB_PATH)
            or os.path.getmtime(LIB_PATH) < os.path.getmtime(src)):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-std=c11", "-fopenmp",
                               "-o", LIB_PATH, src])
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build_oracle_lib())
        u64, p = ctypes.c_uint64, ctypes.c_void_p
        _lib.kor_sanity_check.restype = u64
        _lib.kor_sanity_check.argtypes = [ctypes.c_int, u64, p, p, p, p]
        _lib.kor_process.restype = u64
        _lib.kor_process.argtypes = [ctypes.c_int, u64, p, p, p, p,
                                     ctypes.c_uint32, ctypes.c_int, p, p,
                                     p, p, u64, p, u64]
        _lib.kor_pagerank_f64.restype = None
        _lib.kor_pagerank_f64.argtypes = [u64, p, p, p, ctypes.c_uint32,
                                          ctypes.c_double, p, p]
        _lib.kor_jacobi_fixed_point.restype = u64
        _lib.kor_jacobi_fixed_point.argtypes = [ctypes.c_int, u64, p, p, p,
                                                p, p]
        _lib.kor_gen_rmat.restype = ctypes.c_int
        _lib.kor_gen_rmat.argtypes = [ctypes.c_uint32, u64, u64, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, u64,
                                      ctypes.c_uint32, ctypes.c_uint32, p, p, p]
        _lib.kor_csc_from_edges.restype = ctypes.c_int
        _lib.kor_csc_from_edges.argtypes = [u64, u64, p, p, p, p, p, p]
        _lib.kor_cc_union_find.restype = None
        _lib.kor_cc_union_find.argtypes = [u64, u64, p, p, p]
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


# --------------------------------------------------------------------------
# Host graph construction (graph_raw.h:57-190, graph_csr.h:44-110)
# --------------------------------------------------------------------------

@dataclass
class HostGraph:
    """Fields named after kites::graph_csr's public members (graph_csr.h:28-39)."""
    V: np.ndarray            # uint32 [n_vertices]       (padded to 128)
    R: np.ndarray            # uint64 [n_vertices + 1]   CSC keyed by destination
    C: np.ndarray            # uint32 [n_edges]          sources, sorted per row
    E: np.ndarray            # uint32 [n_edges]
    vBitmap: np.ndarray      # uint32 [ceil(nbits/32)]   initial frontier
    nbits: int
    directed: bool
    vertexPerGroup: int
    dir_R: np.ndarray = field(default_factory=lambda: np.zeros(1, np.uint64))
    dir_C: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    n_unpadded: int = 0

    @property
    def n_vertices(self) -> int:
        return int(self.V.shape[0])

    @property
    def n_edges(self) -> int:
        return int(self.C.shape[0])


def _pack_bits(flags: np.ndarray) -> np.ndarray:
    """bool[n] -> uint32 words, bit i of word w = flag[32 w + i] (LSB first,
    host_pinned_buffer.cuh:151-153)."""
    n = flags.shape[0]
    nw = (n + 31) // 32
    padded = np.zeros(nw * 32, dtype=np.uint8)
    padded[:n] = flags
    return np.packbits(padded.reshape(-1, 8), axis=1,
                       bitorder="little").reshape(-1).view(np.uint32).copy()


def unpack_bits(words: np.ndarray, nbits: int) -> np.ndarray:
    b = np.unpackbits(words.view(np.uint8), bitorder="little")
    return b[:nbits].astype(bool)


def build_host_graph(first, second, weights=None, *, form_s_d=True, vpg=1,
                     directed=True, incomplete=False, init="source",
                     source=0, inf=INF32, weight_rule=None):
    """Build a host graph the way kites::graph_csr's edge-list constructors do.

    first/second: the two columns of the edge list in file order.
    weights: per-line edge values, or None (then ``weight_rule(s, d)``).
    init: the pre-processing function's value rule --
        "source": V[x] = 0 if x == source else inf, activation bit of the
                  destination group set iff the edge's source is ``source``
                  (examples/sssp_basic_single_device.cu:9-27);
        "label":  V[x] = x, every destination activated (min-label CC).
    Vertices that never appear in an edge keep the value-initialised 0
    (graph_raw.h:90-93).  Rows are sorted by source with ties kept in file
    order (the reference's std::sort leaves the order of equal sources
    unspecified; generated graphs have no equal pairs).
    """
    first = np.asarray(first, dtype=np.uint32)
    second = np.asarray(second, dtype=np.uint32)
    ne_in = first.shape[0]
    if form_s_d:
        src, dst = first, second
    else:
        src, dst = second, first
    if weights is None:
        if weight_rule is None:
            w = np.ones(ne_in, dtype=np.uint32)
        else:
            w = weight_rule(src, dst).astype(np.uint32)
    else:
        w = np.asarray(weights, dtype=np.uint32)

    maxid = int(max(first.max(initial=0), second.max(initial=0)))
    n = max(1, maxid + 1)                  # rawVVec starts with one element
    ngroups = -(-n // vpg)

    def value_of(x):
        if init == "source":
            return np.where(x == source, 0, inf).astype(np.uint32)
        if init == "label":
            return x.astype(np.uint32)
        raise ValueError(init)

    def activates(s, d):
        if init == "source":
            return s == source
        return np.ones(s.shape[0], dtype=bool)

    V = np.zeros(n, dtype=np.uint32)
    touched = np.unique(np.concatenate([src, dst]))
    V[touched] = value_of(touched)

    act = np.zeros(ngroups, dtype=bool)
    fire = activates(src, dst)
    act[(dst[fire] // vpg)] = True

    rows_dst, rows_src, rows_w, order_key = dst, src, w, np.arange(ne_in)
    if (not directed) and incomplete:
        fire2 = activates(dst, src)
        act[(src[fire2] // vpg)] = True
        # graph_raw.h:111-121 -- the reverse edge is pushed right after the
        # forward one, with its own pre-processing call.
        # That call sees the endpoints swapped, so a rule-derived value is
        # computed for (dst, src); a value read from the file is the same.
        w_rev = w if (weights is not None or weight_rule is None) else \
            weight_rule(dst, src).astype(np.uint32)
        rows_dst = np.concatenate([dst, src])
        rows_src = np.concatenate([src, dst])
        rows_w = np.concatenate([w, w_rev])
        order_key = np.concatenate([2 * np.arange(ne_in), 2 * np.arange(ne_in) + 1])

    order = np.lexsort((order_key, rows_src, rows_dst))
    C = rows_src[order].astype(np.uint32)
    E = rows_w[order].astype(np.uint32)
    deg = np.bincount(rows_dst, minlength=n).astype(np.uint64)

    n_pad = n if n % 128 == 0 else (n // 128 + 1) * 128
    Vp = np.zeros(n_pad, dtype=np.uint32)
    Vp[:n] = V
    R = np.zeros(n_pad + 1, dtype=np.uint64)
    np.cumsum(deg, out=R[1:n + 1])
    R[n + 1:] = R[n]

    # Initial frontier and group out-adjacency (graph_raw.h:126-181,
    # graph_csr.h:100-108).
    if directed:
        n_out_groups = ngroups
        if vpg == 1:
            o = np.lexsort((dst, src))
            dir_C = dst[o].astype(np.uint32)
            counts = np.bincount(src, minlength=n).astype(np.uint64)
            n_out_groups = n_pad
            dir_counts = np.zeros(n_pad, dtype=np.uint64)
            dir_counts[:n] = counts
            nbits = n_pad
        else:
            pairs = np.unique((src // vpg).astype(np.uint64) << np.uint64(32)
                              | (dst // vpg).astype(np.uint64))
            gs = (pairs >> np.uint64(32)).astype(np.int64)
            dir_C = (pairs & np.uint64(0xFFFFFFFF)).astype(np.uint32)
            dir_counts = np.bincount(gs, minlength=ngroups).astype(np.uint64)
            nbits = ngroups
        dir_R = np.zeros(n_out_groups + 1, dtype=np.uint64)
        np.cumsum(dir_counts, out=dir_R[1:])
        flags = np.zeros(nbits, dtype=bool)
        flags[:ngroups] = act
        # graph_csr.h:100-104 copies bits only for groups < rawIVecOutgoing.size()
        flags[n_out_groups:] = False
    else:
        # dir_R / dir_C are never allocated for undirected graphs.
        dir_R = np.zeros(0, dtype=np.uint64)
        dir_C = np.zeros(0, dtype=np.uint32)
        nbits = ngroups
        # rawIVecOutgoing stays empty for undirected graphs, so no bit is
        # ever copied into graph_csr::vBitmap (graph_csr.h:100-101).
        flags = np.zeros(nbits, dtype=bool)
    return HostGraph(V=Vp, R=R, C=C, E=E, vBitmap=_pack_bits(flags),
                     nbits=int(nbits), directed=directed, vertexPerGroup=vpg,
                     dir_R=dir_R, dir_C=dir_C, n_unpadded=n)


def mipmap_of(hg: HostGraph, cr: int):
    """The block structures kites::graph_csr_mipmapped adds to a directed
    one-vertex-per-group host graph (graph_csr_mipmapped.hpp:40-78):
    mipmapDim = ceil(n / cr) rounded up to a multiple of 32 (n the padded
    vertex count); the block frontier, bit v // cr set for every vertex v
    whose frontier bit is set; the mipmap, a mipmapDim x mipmapDim row-major
    bit matrix with bit (s // cr) * mipmapDim + d // cr set for every edge
    s -> d.  Returns (mipmapDim, frontier words, mipmap words)."""
    assert hg.directed and hg.vertexPerGroup == 1 and cr > 0
    n = hg.n_vertices
    act = np.flatnonzero(unpack_bits(hg.vBitmap, hg.nbits)[:n])
    counts = np.diff(hg.dir_R.astype(np.int64))
    src = np.repeat(np.arange(n, dtype=np.int64), counts)
    dim, words = mipmap_from_edges(n, src, hg.dir_C, cr)
    blocks = np.zeros(dim, dtype=bool)
    blocks[act // cr] = True
    return dim, _pack_bits(blocks), words


def mipmap_from_edges(n: int, src, dst, cr: int):
    """The mipmap of mipmap_of for an edge list s -> d over n vertices:
    (mipmapDim, dim * dim / 32 words), bit (s // cr) * dim + d // cr
    (graph_csr_mipmapped.hpp:58-75)."""
    dim = -(-n // cr)
    dim = -(-dim // 32) * 32
    bit = (np.asarray(src, dtype=np.int64) // cr) * dim + np.asarray(dst, dtype=np.int64) // cr
    words = np.zeros(dim * dim // 32, dtype=np.uint32)
    bit = np.unique(bit)
    np.bitwise_or.at(words, bit >> 5, (np.uint32(1) << (bit & 31).astype(np.uint32)))
    return dim, words


def example_weight_rule(src, dst):
    """(s+1)(d+2) % 127 in uint32 arithmetic
    (examples/sssp_basic_single_device.cu:22-25)."""
    s = src.astype(np.uint64) + 1
    d = dst.astype(np.uint64) + 2
    return ((s * d) & np.uint64(0xFFFFFFFF)) % np.uint64(127)


def read_edge_list(path):
    """Parse an edge list the way graph_raw.h:73-123 does: lines not starting
    with a digit are skipped; the first two whitespace-separated fields are
    the indices; a third field, if present, is the edge value (atoi)."""
    firsts, seconds, extra = [], [], []
    has_weight = False
    with open(path, "r") as f:
        for line in f:
            if not line or line[0] < "0" or line[0] > "9":
                continue
            parts = line.split()
            if len(parts) < 2:
                continue
            firsts.append(int(parts[0]))
            seconds.append(int(parts[1]))
            if len(parts) > 2:
                has_weight = True
                extra.append(int(parts[2]))
            else:
                extra.append(None)
    first = np.array(firsts, dtype=np.uint32)
    second = np.array(seconds, dtype=np.uint32)
    w = None
    if has_weight:
        if any(x is None for x in extra):
            raise ValueError("mixed weighted/unweighted lines")
        w = np.array(extra, dtype=np.uint32)
    return first, second, w


# --------------------------------------------------------------------------
# Fixed points
# --------------------------------------------------------------------------

def gen_rmat(scale, n_edges, a=0.57, b=0.19, c=0.19, seed=1, w_lo=1, w_hi=255,
             n_vertices=0):
    """The benchmark's R-MAT edge list from the oracle's own restatement of
    the generator rule (kor_gen_rmat): same (src, dst, w) as the product's
    generator for the same arguments."""
    src = np.empty(n_edges, dtype=np.uint32)
    dst = np.empty(n_edges, dtype=np.uint32)
    w = np.empty(n_edges, dtype=np.uint32)
    if lib().kor_gen_rmat(scale, n_vertices, n_edges, a, b, c, seed, w_lo, w_hi, _ptr(src),
                          _ptr(dst), _ptr(w)) != 0:
        raise MemoryError("kor_gen_rmat failed")
    return src, dst, w


def csc_from_edges(n_vertices, src, dst, w=None):
    """CSC (rows = destinations, sources ascending, ties in input order) of
    an edge list, by the oracle's own builder (kor_csc_from_edges)."""
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    m = src.shape[0]
    R = np.empty(n_vertices + 1, dtype=np.uint64)
    C = np.empty(m, dtype=np.uint32)
    E = np.empty(m, dtype=np.uint32) if w is not None else None
    w = None if w is None else np.ascontiguousarray(w, dtype=np.uint32)
    if lib().kor_csc_from_edges(n_vertices, m, _ptr(src), _ptr(dst), _ptr(w), _ptr(R),
                                _ptr(C), _ptr(E)) != 0:
        raise ValueError("kor_csc_from_edges failed (bad endpoint or out of memory)")
    return R, C, E


def sanity_check(hg_or_R, C=None, E=None, V=None, op=OP_SSSP_SAT):
    """Gauss-Seidel fixed point (sanity_check.cuh:22-47). Returns (V, sweeps)."""
    if isinstance(hg_or_R, HostGraph):
        R, C, E, V = hg_or_R.R, hg_or_R.C, hg_or_R.E, hg_or_R.V
    else:
        R = hg_or_R
    R = np.ascontiguousarray(R, dtype=np.uint64)
    C = np.ascontiguousarray(C, dtype=np.uint32)
    Ea = None if E is None else np.ascontiguousarray(E, dtype=np.uint32)
    out = np.array(V, dtype=np.uint32, copy=True)
    sweeps = lib().kor_sanity_check(op, out.shape[0], _ptr(R), _ptr(C),
                                    _ptr(Ea), _ptr(out))
    return out, int(sweeps)


def jacobi_fixed_point(R, C, E, V, op=OP_SSSP_SAT):
    R = np.ascontiguousarray(R, dtype=np.uint64)
    C = np.ascontiguousarray(C, dtype=np.uint32)
    Ea = None if E is None else np.ascontiguousarray(E, dtype=np.uint32)
    out = np.array(V, dtype=np.uint32, copy=True)
    nxt = np.empty_like(out)
    rounds = lib().kor_jacobi_fixed_point(op, out.shape[0], _ptr(R), _ptr(C),
                                          _ptr(Ea), _ptr(out), _ptr(nxt))
    return out, int(rounds)


def process(hg: HostGraph, op=OP_SSSP_SAT, max_iterations=1 << 40):
    """Sequential restatement of kites::process (compute.cuh:29-137)."""
    V = hg.V.copy()
    nw = (hg.nbits + 31) // 32
    even = np.zeros(max(nw, 1), dtype=np.uint32)
    even[:hg.vBitmap.shape[0]] = hg.vBitmap
    odd = np.zeros_like(even)
    ngroups = -(-hg.n_vertices // hg.vertexPerGroup)
    scratch = np.zeros(max(ngroups, 1), dtype=np.uint32)
    dir_R = np.ascontiguousarray(hg.dir_R, dtype=np.uint64)
    dir_C = np.ascontiguousarray(hg.dir_C, dtype=np.uint32)
    if dir_C.shape[0] == 0:
        dir_C = np.zeros(1, dtype=np.uint32)
    iters = lib().kor_process(op, hg.n_vertices, _ptr(hg.R), _ptr(hg.C),
                              _ptr(hg.E), _ptr(V), hg.vertexPerGroup,
                              1 if hg.directed else 0, _ptr(dir_R),
                              _ptr(dir_C), _ptr(even), _ptr(odd),
                              hg.nbits, _ptr(scratch), max_iterations)
    return V, int(iters)


def pagerank_f64(n_real, R, C, out_degree, iterations=20, damping=0.85):
    R = np.ascontiguousarray(R, dtype=np.uint64)
    C = np.ascontiguousarray(C, dtype=np.uint32)
    od = np.ascontiguousarray(out_degree, dtype=np.uint32)
    pr = np.zeros(n_real, dtype=np.float64)
    tmp = np.zeros(n_real, dtype=np.float64)
    lib().kor_pagerank_f64(n_real, _ptr(R), _ptr(C), _ptr(od), iterations,
                           damping, _ptr(pr), _ptr(tmp))
    return pr


# --------------------------------------------------------------------------
# Size-independent certificates (numpy, vectorised)
# --------------------------------------------------------------------------

def _sat_add(a, b):
    s = a.astype(np.uint64) + b.astype(np.uint64)
    return np.minimum(s, np.uint64(INF32)).astype(np.uint32)


def _row_ids(R):
    deg = np.diff(R.astype(np.int64))
    return np.repeat(np.arange(deg.shape[0], dtype=np.int64), deg)


def certify_shortest_paths(R, C, E, dist, sources_zero, unit_weight=False):
    """True iff ``dist`` is the unique shortest-path fixed point from the
    vertices in ``sources_zero`` (positive weights): (1) sources hold 0;
    (2) no edge relaxes (dist[v] <= dist[u] + w); (3) every other finite
    vertex has a tight in-edge.  Returns (ok, message)."""
    dist = np.asarray(dist, dtype=np.uint32)
    if np.any(dist[np.asarray(sources_zero, dtype=np.int64)] != 0):
        return False, "source distance is not 0"
    v_of_e = _row_ids(R)
    w = np.ones_like(C) if unit_weight else E
    cand = _sat_add(dist[C], w)
    if np.any(cand < dist[v_of_e]):
        bad = int(np.argmax(cand < dist[v_of_e]))
        return False, f"edge {bad} relaxes vertex {int(v_of_e[bad])}"
    tight = (cand == dist[v_of_e]) & (cand != INF32)
    has_tight = np.zeros(dist.shape[0], dtype=bool)
    has_tight[v_of_e[tight]] = True
    is_src = np.zeros(dist.shape[0], dtype=bool)
    is_src[np.asarray(sources_zero, dtype=np.int64)] = True
    need = (dist != INF32) & ~is_src
    if np.any(need & ~has_tight):
        bad = int(np.argmax(need & ~has_tight))
        return False, f"vertex {bad} finite without a tight in-edge"
    return True, "ok"


def cc_min_labels(n_vertices, src, dst):
    """Exact min-label CC of the undirected graph behind an edge list (each
    edge in both directions): the smallest vertex id of every vertex's
    component, by union-find (kor_cc_union_find)."""
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    out = np.empty(n_vertices, dtype=np.uint32)
    lib().kor_cc_union_find(n_vertices, src.shape[0], _ptr(src), _ptr(dst), _ptr(out))
    return out


def certify_min_label(R, C, labels):
    """Min-label CC certificate on a symmetric graph: labels equal across
    every edge, label[v] <= v, and label[label[v]] == label[v]."""
    labels = np.asarray(labels, dtype=np.uint32)
    v_of_e = _row_ids(R)
    if np.any(labels[C] != labels[v_of_e]):
        return False, "edge with differing labels"
    idx = np.arange(labels.shape[0], dtype=np.uint64)
    if np.any(labels.astype(np.uint64) > idx):
        return False, "label above own id"
    if np.any(labels[labels] != labels):
        return False, "label root does not label itself"
    return True, "ok"
