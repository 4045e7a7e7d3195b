"""Full-size runs of the scale-22 configuration: a directed R-MAT graph of
scale 22 (4,194,304 vertices, 67,108,864 edges, a,b,c = 0.57,0.19,0.19,
uint32 weights U[1,255]) and an Erdos-Renyi graph with the same V and E.
On each: plain SSSP and BFS from 8 seeded sources (checked by the
shortest-path certificate, which only the unique fixed point passes),
min-label CC on the symmetrised graph (every edge in both directions, as
the reference's undirected construction lists them) against the oracle's
exact union-find labels, and the vertex-per-group sweep {1, 2, 4, 8}: the
group graphs (activation by deduplicated group adjacency,
kites/device/kernels_single_device.cuh:174-426) reach bit-identical
distances and levels."""
import numpy as np
import pytest

from kites_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N = 1 << 22
M = 16 * N


def seeded_sources(outdeg, count, seed):
    cand = np.flatnonzero(outdeg > 0)
    rng = np.random.default_rng(seed)
    return [int(v) for v in rng.choice(cand, size=count, replace=False)]


@pytest.fixture(scope="module", params=["rmat22", "er22"])
def graph22(request, engine):
    if request.param == "rmat22":
        s, d, w = capi.gen_rmat(22, M, 0.57, 0.19, 0.19, seed=1, w_lo=1, w_hi=255)
    else:
        s, d, w = capi.gen_er(N, M, seed=1, w_lo=1, w_hi=255)
    R, C, E = capi.csc_from_edges(N, s, d, w)
    g = capi.Graph(engine, R, C, E)
    srcs = seeded_sources(np.bincount(s, minlength=N), 8, 22)
    yield request.param, s, d, R, C, E, g, srcs
    g.close()


def test_sssp_and_bfs_from_8_sources(graph22):
    name, s, d, R, C, E, g, srcs = graph22
    for src in srcs:
        dist, st = g.sssp(src)
        ok, msg = O.certify_shortest_paths(R, C, E, dist, [src])
        assert ok, f"{name} SSSP from {src}: {msg}"
        assert st.iterations > 1
        lev, _ = g.sssp(src, op=capi.OP_BFS)
        ok, msg = O.certify_shortest_paths(R, C, E, lev, [src], unit_weight=True)
        assert ok, f"{name} BFS from {src}: {msg}"


def test_cc_on_symmetrised_graph(graph22, engine):
    name, s, d, R, C, E, g, srcs = graph22
    gs = capi.Graph.from_edges(engine, N, np.concatenate([s, d]), np.concatenate([d, s]),
                               directed=False)
    try:
        labels, st = gs.cc()
        np.testing.assert_array_equal(labels, O.cc_min_labels(N, s, d))
        assert st.iterations > 1
    finally:
        gs.close()


def group_adjacency(s, d, vpg):
    """Deduplicated (source group -> destination group) adjacency, rows by
    source group (graph_raw.h:126-181)."""
    shift = vpg.bit_length() - 1
    key = np.unique((s >> shift).astype(np.uint64) << np.uint64(32) | (d >> shift))
    rows = (key >> np.uint64(32)).astype(np.int64)
    dir_C = (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    dir_R = np.zeros(N // vpg + 1, np.uint64)
    np.cumsum(np.bincount(rows, minlength=N // vpg), out=dir_R[1:])
    return dir_R, dir_C


@pytest.mark.parametrize("vpg", [2, 4, 8])
def test_vertex_per_group_sweep(graph22, engine, vpg):
    name, s, d, R, C, E, g, srcs = graph22
    dir_R, dir_C = group_adjacency(s, d, vpg)
    gv = capi.Graph(engine, R, C, E, vpg=vpg, dir_R=dir_R, dir_C=dir_C)
    try:
        assert gv.device_view().vertex_per_group == vpg
        for src in srcs:
            for op in (capi.OP_SSSP, capi.OP_BFS):
                want, _ = g.sssp(src, op=op)
                got, _ = gv.sssp(src, op=op)
                np.testing.assert_array_equal(got, want, err_msg=f"{name} vpg {vpg} src {src}")
    finally:
        gv.close()
