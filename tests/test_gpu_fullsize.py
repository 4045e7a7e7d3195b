"""Full-size parity through size-independent certificates (R-MAT scale 22,
67M edges): the oracle's sequential loop is too slow here, so each result
is checked as the unique fixed point it must be."""
import ctypes

import numpy as np
import pytest

from kites_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rmat22(engine):
    n = 1 << 22
    s, d, w = capi.gen_rmat(22, 16 * n, seed=1)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    del s, d, w
    g = capi.Graph(engine, R, C, E)
    yield g, R, C, E, n
    g.close()


@pytest.mark.parametrize("strategy", [capi.STRATEGY_PLAIN, capi.STRATEGY_AUTO,
                                      capi.STRATEGY_PUSH, capi.STRATEGY_PULL_ALL])
def test_scale22_single_source(rmat22, strategy):
    g, R, C, E, n = rmat22
    for src in (0, 123457):
        dist, st = g.sssp(src, opts=capi.default_opts(strategy=strategy))
        ok, msg = O.certify_shortest_paths(R, C, E, dist, [src])
        assert ok, msg
        assert (dist != O.INF32).sum() > n // 4


def test_scale22_bfs(rmat22):
    g, R, C, E, n = rmat22
    dist, _ = g.sssp(5, op=capi.OP_BFS)
    ok, msg = O.certify_shortest_paths(R, C, E, dist, [5], unit_weight=True)
    assert ok, msg


@pytest.mark.parametrize("k", [64, 256])
def test_scale22_batched(rmat22, k):
    g, R, C, E, n = rmat22
    srcs = np.random.default_rng(k).choice(n, size=k, replace=False).astype(np.uint32)
    dist = np.empty((n, k), np.uint32)
    st = capi.RunStats()
    o = capi.default_opts()
    capi._check(capi.load().kites_sssp_batch(g.engine._h, g._h, capi.OP_SSSP, capi._p(srcs), k,
                                             capi._p(dist), ctypes.byref(o), ctypes.byref(st)))
    for j in range(0, k, k // 8):
        ok, msg = O.certify_shortest_paths(R, C, E, dist[:, j], [int(srcs[j])])
        assert ok, f"slot {j}: {msg}"
    # One column against the single-source kernel, bit for bit.
    single, _ = g.sssp(int(srcs[3]))
    np.testing.assert_array_equal(dist[:, 3], single)
