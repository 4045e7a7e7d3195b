"""The mipmapped frontier as an engine strategy: the block map built on the
device equals kites::graph_csr_mipmapped's (graph_csr_mipmapped.hpp:58-75,
through the oracle pinned to the reference's class and, for config 1, the
reference's own golden hashes), and KITES_STRATEGY_MIP -- alone, as the
selector's coarse class, and through the autotuner -- reaches the oracle's
fixed point bit for bit."""
import numpy as np
import pytest

from kites_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

INF = O.INF32
BLOCKS = [1, 3, 32, 100, 1024]


def graphs():
    s, d, w = capi.gen_rmat(12, 16 << 12, seed=41)
    yield "rmat12", 1 << 12, s, d, w
    s, d, w = capi.gen_grid(40, seed=5)          # 1,600 vertices: padded to 1,664
    yield "grid40", 40 * 40, s, d, w
    s, d, w = capi.gen_er(3000, 20000, seed=6)
    yield "er3k", 3000, s, d, w


GRAPHS = list(graphs())


@pytest.fixture(scope="module")
def uploaded(engine):
    out = {}
    for name, n, s, d, w in GRAPHS:
        R, C, E = capi.csc_from_edges(n, s, d, w)
        out[name] = (capi.Graph(engine, R, C, E), R, C, E, n, s, d)
    yield out
    for g, *_ in out.values():
        g.close()


def padded(n):
    return -(-n // 128) * 128


@pytest.mark.parametrize("block", BLOCKS)
@pytest.mark.parametrize("name", [g[0] for g in GRAPHS])
def test_block_map_matches_oracle(uploaded, name, block):
    g, R, C, E, n, s, d = uploaded[name]
    g.build_mipmap(block)
    dim, words = g.mipmap()
    want_dim, want = O.mipmap_from_edges(padded(n), s, d, block)
    assert dim == want_dim
    np.testing.assert_array_equal(words, want)


@pytest.mark.parametrize("cr", [1, 3, 32, 100])
def test_block_map_matches_reference_cfg1(engine, golden, cfg1_edges, cr):
    """Config 1 (7,115 vertices, padded to 7,168): the engine's map and dim
    against the reference class's own (golden dim, and the map equal to the
    oracle's, whose hash the reference's class pins in the CPU tests)."""
    s, d, w = cfg1_edges
    R, C, E = capi.csc_from_edges(7115, s, d, w)
    g = capi.Graph(engine, R, C, E)
    try:
        g.build_mipmap(cr)
        dim, words = g.mipmap()
        assert dim == golden["meta"]["cfg1_mipmap_dim"][str(cr)]
        hg = O.build_host_graph(s, d, w, init="source", source=0, inf=(1 << 30) - 1)
        _, _, mip = O.mipmap_of(hg, cr)
        np.testing.assert_array_equal(words, mip)
    finally:
        g.close()


@pytest.mark.parametrize("block", [1, 32, 100, 1024])
@pytest.mark.parametrize("device_loop", [0, 1])
@pytest.mark.parametrize("name", [g[0] for g in GRAPHS])
def test_mip_strategy_sssp_bfs(uploaded, name, device_loop, block):
    g, R, C, E, n, s, d = uploaded[name]
    g.build_mipmap(block)
    o = capi.default_opts(strategy=capi.STRATEGY_MIP, device_loop=device_loop)
    for op, oop in [(capi.OP_SSSP, O.OP_SSSP_SAT), (capi.OP_BFS, O.OP_BFS_SAT)]:
        src = 5
        dist, st = g.sssp(src, op=op, opts=o)
        V0 = np.full(n, INF, np.uint32)
        V0[src] = 0
        want, _ = O.sanity_check(R, C, E, V0, op=oop)
        np.testing.assert_array_equal(dist, want)
        assert st.strategy_hist[capi.STRATEGY_MIP] == st.iterations


def test_mip_strategy_cc(engine, cfg1_edges, golden):
    s, d, _ = cfg1_edges
    ss, tt = np.concatenate([s, d]), np.concatenate([d, s])
    k = np.unique(ss.astype(np.uint64) << np.uint64(32) | tt)
    ss = (k >> np.uint64(32)).astype(np.uint32)
    tt = (k & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    R, C, _ = capi.csc_from_edges(7115, ss, tt)
    g = capi.Graph(engine, R, C, None)
    try:
        g.build_mipmap(64)
        labels, st = g.cc(opts=capi.default_opts(strategy=capi.STRATEGY_MIP))
        np.testing.assert_array_equal(labels, golden["cfg1_cc"][:7115])
        assert st.strategy_hist[capi.STRATEGY_MIP] == st.iterations
    finally:
        g.close()


def coarse_selector():
    """Selector weights that always predict class 2 (coarse) far below PLAIN."""
    P = np.zeros(capi.SELECTOR_PARAMS, np.float32)
    P[capi.SEL_OFF["std"]:capi.SEL_OFF["std"] + 12] = 1.0
    P[capi.SEL_OFF["b3"] + 2] = -5.0
    return P


def test_coarse_class_runs_mip(engine, uploaded):
    g, R, C, E, n, s, d = uploaded["grid40"]
    saved = engine.selector_save()
    try:
        engine.selector_load(coarse_selector())
        g.build_mipmap(40)
        g.set_coarse(capi.STRATEGY_MIP)
        o = capi.default_opts(strategy=capi.STRATEGY_AUTO)
        dist, st = g.sssp(3, opts=o)
        V0 = np.full(n, INF, np.uint32)
        V0[3] = 0
        want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
        np.testing.assert_array_equal(dist, want)
        assert st.strategy_hist[capi.STRATEGY_MIP] == st.iterations
        g.set_coarse(capi.STRATEGY_PULL_ALL)
        dist, st = g.sssp(3, opts=o)
        np.testing.assert_array_equal(dist, want)
        assert st.strategy_hist[capi.STRATEGY_PULL_ALL] == st.iterations
    finally:
        engine.selector_load(saved)
        g.set_coarse(capi.STRATEGY_PULL_ALL)


def test_autotune_picks_a_coarse_class(engine, uploaded):
    g, R, C, E, n, s, d = uploaded["rmat12"]
    g.build_mipmap(32)
    r = g.autotune(np.array([1, 2, 3, 4], np.uint32), batch=0)
    assert r.coarse_strategy in (capi.STRATEGY_PULL_ALL, capi.STRATEGY_MIP)
    assert r.coarse_ms > 0
    dist, _ = g.sssp(9, opts=capi.default_opts(strategy=capi.STRATEGY_AUTO))
    V0 = np.full(n, INF, np.uint32)
    V0[9] = 0
    want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
    np.testing.assert_array_equal(dist, want)
    g.set_coarse(capi.STRATEGY_PULL_ALL)


def test_mip_errors(engine):
    s, d, w = capi.gen_er(2000, 8000, seed=9)
    R, C, E = capi.csc_from_edges(2000, s, d, w)
    g = capi.Graph(engine, R, C, E)
    try:
        with pytest.raises(capi.KitesError):
            g.sssp(0, opts=capi.default_opts(strategy=capi.STRATEGY_MIP))
        with pytest.raises(capi.KitesError):
            g.set_coarse(capi.STRATEGY_MIP)
        with pytest.raises(capi.KitesError):
            g.set_coarse(capi.STRATEGY_PUSH)
        with pytest.raises(capi.KitesError):
            g.build_mipmap(0)
        with pytest.raises(capi.KitesError):
            g.mipmap()
        # Rebuilding replaces the map.
        g.build_mipmap(16)
        assert g.mipmap()[0] == 128
        g.build_mipmap(1000)
        assert g.mipmap()[0] == 32
    finally:
        g.close()


def test_mip_rejects_an_oversized_map(engine):
    n = 70000                       # padded 70,016 > 65,536 blocks of one vertex
    s = np.arange(n - 1, dtype=np.uint32)
    d = s + 1
    R, C, E = capi.csc_from_edges(n, s, d, np.ones(n - 1, np.uint32))
    g = capi.Graph(engine, R, C, E)
    try:
        with pytest.raises(capi.KitesError):
            g.build_mipmap(1)
        g.build_mipmap(4)           # 17,504 blocks
        assert g.mipmap()[0] == 17504
    finally:
        g.close()
