"""The largest single-GPU case: R-MAT scale 26 (67,108,864 vertices,
1,073,741,824 edges before deduplication, uint32 ids and weights).

The edge list is generated on the host and its CSC is built on the device
(kites_graph_from_edges); a second copy of the graph is uploaded with 64-bit
row offsets, the layout graphs past 2^32 vertices + edges get.  Checked:

* 16-source batched SSSP: the shortest-path certificate (sources 0, no edge
  relaxes, every finite vertex has a tight in-edge) on sampled columns, and
  one column against the single-source plain kernel bit for bit;
* single-source SSSP with the learned selector (AUTO) equal to PLAIN, on
  both offset layouts;
* FP32 PageRank, 20 iterations, damping 0.85, uniform 1/V start, within
  1e-5 relative L1 of the FP64 oracle;
* min-label CC on the symmetrised graph (every edge in both directions,
  2,147,483,648 edges, past 2^31), its CSC built on the device, against the
  oracle's exact union-find labels.

The oracle's sequential loop would take hours here, so distances are judged
by the certificate, which holds only for the unique fixed point."""
import numpy as np
import pytest

from kites_b200 import capi
from oracle import oracle as O
from test_gpu_ingest import csc_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rmat26(engine):
    n = 1 << 26
    s, d, w = capi.gen_rmat(26, 16 * n, seed=1)
    outdeg = np.bincount(s, minlength=n).astype(np.uint32)
    g = capi.Graph.from_edges(engine, n, s, d, w)
    del w
    R, C, E = csc_of(g)
    yield g, R[: n + 1], C, E, outdeg, n, s, d
    g.close()


def test_scale26_batched_sssp(rmat26):
    g, R, C, E, outdeg, n, _, _ = rmat26
    srcs = np.flatnonzero(outdeg > 0)[[0, 1000, 5000, 10**5, 10**6, 3 * 10**6, 5 * 10**6,
                                       7 * 10**6, 9 * 10**6, 11 * 10**6, 13 * 10**6,
                                       15 * 10**6, 17 * 10**6, 19 * 10**6, 21 * 10**6,
                                       23 * 10**6]].astype(np.uint32)
    dist, st = g.sssp_batch(srcs)
    assert dist.shape == (n, 16) and st.iterations > 1
    for j in (0, 9):
        ok, msg = O.certify_shortest_paths(R, C, E, dist[:, j], [int(srcs[j])])
        assert ok, f"slot {j}: {msg}"
    single, _ = g.sssp(int(srcs[9]))
    np.testing.assert_array_equal(dist[:, 9], single)


def test_scale26_auto_equals_plain_on_both_offset_layouts(rmat26, engine):
    g, R, C, E, outdeg, n, _, _ = rmat26
    src = int(np.flatnonzero(outdeg > 0)[12345])
    plain, _ = g.sssp(src)
    auto, st = g.sssp(src, opts=capi.default_opts(strategy=capi.STRATEGY_AUTO))
    np.testing.assert_array_equal(auto, plain)
    assert sum(st.strategy_hist) == st.iterations
    g64 = capi.Graph(engine, R, C, E, offsets64=True)
    assert g64.device_view().offsets64 == 1
    auto64, _ = g64.sssp(src, opts=capi.default_opts(strategy=capi.STRATEGY_AUTO))
    np.testing.assert_array_equal(auto64, plain)
    g64.close()


def test_scale26_pagerank_fp64_oracle(rmat26):
    g, R, C, E, outdeg, n, _, _ = rmat26
    pr, st = g.pagerank(n_real=n, iterations=20, damping=0.85)
    want = O.pagerank_f64(n, R, C, outdeg, 20, 0.85)
    rel_l1 = np.abs(pr.astype(np.float64) - want).sum() / np.abs(want).sum()
    assert rel_l1 < 1e-5, rel_l1
    assert st.iterations == 20


def test_scale26_cc_symmetrised(rmat26, engine):
    """Runs last in this module: the directed graph's device arrays are
    released first, so that the symmetrised graph's build has room."""
    g, R, C, E, outdeg, n, s, d = rmat26
    g.close()
    want = O.cc_min_labels(n, s, d)
    gs = capi.Graph.from_edges(engine, n, np.concatenate([s, d]), np.concatenate([d, s]),
                               directed=False)
    try:
        assert gs.n_edges == 2 * s.shape[0] == 1 << 31  # past the old 2^31 - 1 limit
        labels, st = gs.cc()
        np.testing.assert_array_equal(labels, want)
        assert st.iterations > 1
    finally:
        gs.close()
