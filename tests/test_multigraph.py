"""Multi-graph batches: a disjoint union of independent R-MAT graphs run as
one multi-seed SSSP.  Each member's distances must equal its own
single-source fixed point."""
import numpy as np
import pytest

from kites_b200 import capi
from oracle import oracle as O

INF = O.INF32


def union(n_graphs=40, seed=5, v_max=20000):
    return capi.gen_rmat_union(n_graphs, seed=seed, v_min=1000, v_max=v_max)


def test_union_members_are_standalone_graphs():
    s, d, w, vo, eo = union()
    assert vo.shape[0] == 41 and eo.shape[0] == 41
    member = np.searchsorted(vo, s, side="right") - 1
    assert np.array_equal(member, np.searchsorted(vo, d, side="right") - 1)
    assert not np.any(s == d)
    keys = s.astype(np.uint64) << np.uint64(32) | d
    assert np.unique(keys).shape[0] == keys.shape[0]
    for i in (0, 7, 39):
        nv = int(vo[i + 1] - vo[i])
        scale = int(np.ceil(np.log2(nv)))
        si, di, wi = capi.gen_rmat(scale, int(eo[i + 1] - eo[i]), seed=5 * 1000003 + i,
                                   n_vertices=nv)
        lo, hi = int(eo[i]), int(eo[i + 1])
        assert np.array_equal(s[lo:hi] - vo[i], si)
        assert np.array_equal(d[lo:hi] - vo[i], di)
        assert np.array_equal(w[lo:hi], wi)
    # Vertex counts log-uniform in [1000, 20000], edge factors in [4, 32].
    nv = np.diff(vo)
    ef = np.diff(eo) // nv
    assert nv.min() >= 1000 and nv.max() <= 20000
    assert ef.min() >= 4 and ef.max() <= 32


@pytest.mark.gpu
@pytest.mark.parametrize("strategy", [capi.STRATEGY_PLAIN, capi.STRATEGY_AUTO,
                                      capi.STRATEGY_PUSH])
def test_multigraph_batch_matches_members(engine, strategy):
    s, d, w, vo, eo = union()
    n = int(vo[-1])
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(engine, R, C, E)
    seeds = vo[:-1].astype(np.uint32)  # vertex 0 of every member
    dist, st = g.sssp_multi_seed(seeds, opts=capi.default_opts(strategy=strategy))
    for i in (0, 3, 17, 39):
        lo, hi = int(vo[i]), int(vo[i + 1])
        el, eh = int(eo[i]), int(eo[i + 1])
        Ri, Ci, Ei = capi.csc_from_edges(hi - lo, s[el:eh] - lo, d[el:eh] - lo, w[el:eh])
        V0 = np.full(hi - lo, INF, np.uint32)
        V0[0] = 0
        want, _ = O.sanity_check(Ri, Ci, Ei, V0, op=O.OP_SSSP_SAT)
        np.testing.assert_array_equal(dist[lo:hi], want, err_msg=f"member {i}")
    # Full-size certificate over the whole union.
    ok, msg = O.certify_shortest_paths(R, C, E, dist, seeds)
    assert ok, msg


@pytest.mark.gpu
def test_thousand_graph_batch(engine):
    """The full multi-graph batch: 1,000 independent R-MAT graphs, vertex
    counts log-uniform in [1K, 100K], edge factors in [4, 32], vertex 0 of
    every member as its seed, one run of the CUDA-graph device loop with the
    learned selector.  Every member's distances form its own shortest-path
    fixed point (certificate over the whole union) and sampled members match
    the oracle's sequential loop."""
    s, d, w, vo, eo = capi.gen_rmat_union(1000, seed=11, v_min=1000, v_max=100000)
    n = int(vo[-1])
    assert vo.shape[0] == 1001
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(engine, R, C, E)
    seeds = vo[:-1].astype(np.uint32)
    dist, st = g.sssp_multi_seed(seeds, opts=capi.default_opts(strategy=capi.STRATEGY_AUTO))
    ok, msg = O.certify_shortest_paths(R, C, E, dist, seeds)
    assert ok, msg
    plain, _ = g.sssp_multi_seed(seeds)
    np.testing.assert_array_equal(dist, plain)
    for i in (0, 499, 999):
        lo, hi = int(vo[i]), int(vo[i + 1])
        el, eh = int(eo[i]), int(eo[i + 1])
        Ri, Ci, Ei = capi.csc_from_edges(hi - lo, s[el:eh] - lo, d[el:eh] - lo, w[el:eh])
        V0 = np.full(hi - lo, INF, np.uint32)
        V0[0] = 0
        want, _ = O.sanity_check(Ri, Ci, Ei, V0, op=O.OP_SSSP_SAT)
        np.testing.assert_array_equal(dist[lo:hi], want, err_msg=f"member {i}")
    g.close()
