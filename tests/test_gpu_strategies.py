"""Per-iteration strategies and the learned selector: every strategy, and
every mix of strategies the selector picks, reaches the oracle's fixed
point bit for bit."""
import numpy as np
import pytest

from kites_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

INF = O.INF32
STRATEGIES = [capi.STRATEGY_PLAIN, capi.STRATEGY_PUSH, capi.STRATEGY_PULL_ALL,
              capi.STRATEGY_TPV1, capi.STRATEGY_TPV4, capi.STRATEGY_TPV8,
              capi.STRATEGY_TPV32, capi.STRATEGY_AUTO]


def graphs():
    s, d, w = capi.gen_rmat(14, 16 << 14, seed=31)
    yield "rmat14", 1 << 14, s, d, w
    s, d, w = capi.gen_grid(48, seed=3)
    yield "grid48", 48 * 48, s, d, w
    s, d, w = capi.gen_er(5000, 30000, seed=4)
    yield "er5k", 5000, s, d, w


GRAPHS = list(graphs())


@pytest.fixture(scope="module")
def uploaded(engine):
    out = {}
    for name, n, s, d, w in GRAPHS:
        R, C, E = capi.csc_from_edges(n, s, d, w)
        out[name] = (capi.Graph(engine, R, C, E), R, C, E, n)
    yield out
    for g, *_ in out.values():
        g.close()


@pytest.mark.parametrize("strategy", STRATEGIES)
@pytest.mark.parametrize("device_loop", [0, 1])
@pytest.mark.parametrize("name", [g[0] for g in GRAPHS])
def test_strategy_sssp_bfs(uploaded, strategy, device_loop, name):
    g, R, C, E, n = uploaded[name]
    o = capi.default_opts(strategy=strategy, device_loop=device_loop)
    for op, oop in [(capi.OP_SSSP, O.OP_SSSP_SAT), (capi.OP_BFS, O.OP_BFS_SAT)]:
        src = 7
        dist, st = g.sssp(src, op=op, opts=o)
        V0 = np.full(n, INF, np.uint32)
        V0[src] = 0
        want, _ = O.sanity_check(R, C, E, V0, op=oop)
        np.testing.assert_array_equal(dist, want)
        assert sum(st.strategy_hist) == st.iterations


@pytest.mark.parametrize("strategy", [capi.STRATEGY_PUSH, capi.STRATEGY_PULL_ALL,
                                      capi.STRATEGY_TPV8, capi.STRATEGY_AUTO])
def test_strategy_cc(engine, cfg1_edges, golden, strategy):
    s, d, _ = cfg1_edges
    ss, tt = np.concatenate([s, d]), np.concatenate([d, s])
    k = np.unique(ss.astype(np.uint64) << np.uint64(32) | tt)
    ss = (k >> np.uint64(32)).astype(np.uint32)
    tt = (k & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    R, C, _ = capi.csc_from_edges(7115, ss, tt)
    g = capi.Graph(engine, R, C, None)
    labels, _ = g.cc(opts=capi.default_opts(strategy=strategy))
    np.testing.assert_array_equal(labels, golden["cfg1_cc"][:7115])


def forced_selector(cls):
    """Selector weights that always predict class `cls` far below PLAIN."""
    P = np.zeros(capi.SELECTOR_PARAMS, np.float32)
    P[capi.SEL_OFF["std"]:capi.SEL_OFF["std"] + 12] = 1.0
    b3 = capi.SEL_OFF["b3"]
    P[b3:b3 + 4] = 0.0
    if cls:
        P[b3 + cls] = -5.0
    return P


@pytest.mark.parametrize("cls", [0, 1, 2, 3])
@pytest.mark.parametrize("device_loop", [0, 1])
def test_selector_switch_takes_each_class(engine, uploaded, cls, device_loop):
    g, R, C, E, n = uploaded["rmat14"]
    engine.selector_load(forced_selector(cls))
    try:
        o = capi.default_opts(strategy=capi.STRATEGY_AUTO, device_loop=device_loop)
        dist, st = g.sssp(3, opts=o)
        V0 = np.full(n, INF, np.uint32)
        V0[3] = 0
        want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
        np.testing.assert_array_equal(dist, want)
        strat = capi.CLASS_STRATEGY[cls] if cls != 3 else capi.STRATEGY_TPV8
        assert st.strategy_hist[strat] == st.iterations, list(st.strategy_hist)
    finally:
        engine.selector_load(forced_selector(0))


def test_selector_record_train_and_run(engine, uploaded):
    g, R, C, E, n = uploaded["rmat14"]
    X, T = [], []
    for src in (1, 2, 5, 9):
        x, t = g.selector_record(capi.OP_SSSP, src, capacity=256)
        assert x.shape[0] >= 3 and np.all(t > 0)
        X.append(x)
        T.append(t)
    X, T = np.concatenate(X), np.concatenate(T)
    params, loss = engine.selector_train(X, T, epochs=400, lr=3e-3, seed=2)
    assert np.isfinite(loss) and params.shape == (capi.SELECTOR_PARAMS,)
    np.testing.assert_array_equal(engine.selector_save(), params)
    # Whatever it picks, the result is the fixed point.
    o = capi.default_opts(strategy=capi.STRATEGY_AUTO, selector_margin=0.0)
    dist, st = g.sssp(11, opts=o)
    V0 = np.full(n, INF, np.uint32)
    V0[11] = 0
    want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
    np.testing.assert_array_equal(dist, want)
    engine.selector_load(forced_selector(0))


def test_autotune_keeps_results(engine):
    n = 1 << 15
    s, d, w = capi.gen_rmat(15, 16 << 15, seed=41)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(engine, R, C, E)
    srcs = np.array([1, 2, 3, 4], np.uint32)
    r = g.autotune(srcs, batch=16)
    assert r.batch_chunk_items in (128, 256, 512, 1024, 2048)
    assert r.tpv_strategy in (capi.STRATEGY_TPV1, capi.STRATEGY_TPV4, capi.STRATEGY_TPV8,
                              capi.STRATEGY_TPV32)
    assert r.trials > 10 and r.plain_ms > 0 and r.batch_ms > 0
    for strategy in (capi.STRATEGY_PLAIN, capi.STRATEGY_AUTO):
        dist, _ = g.sssp(9, opts=capi.default_opts(strategy=strategy))
        V0 = np.full(n, INF, np.uint32)
        V0[9] = 0
        want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
        np.testing.assert_array_equal(dist, want)
    bd, _ = g.sssp_batch(np.arange(16, dtype=np.uint32) * 7)
    for j in (0, 5):
        V0 = np.full(n, INF, np.uint32)
        V0[j * 7] = 0
        want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
        np.testing.assert_array_equal(bd[:, j], want)


@pytest.mark.parametrize("dense", [0, 1])
def test_plain_sweep_gate_both_paths(engine, dense):
    """Force the plain loop's pull and activation onto the staged sweeps
    (dense) or the chunked kernels (sparse) for every iteration."""
    n = 1 << 14
    s, d, w = capi.gen_rmat(14, 16 << 14, seed=43)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(engine, R, C, E)
    tune = capi.load().kites_graph_set_density
    capi._check(tune(g._h, 0 if dense else 1 << 62, 0 if dense else 1 << 62))
    for strategy in (capi.STRATEGY_PLAIN, capi.STRATEGY_AUTO):
        for dl in (0, 1):
            dist, _ = g.sssp(5, opts=capi.default_opts(strategy=strategy, device_loop=dl))
            V0 = np.full(n, INF, np.uint32)
            V0[5] = 0
            want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
            np.testing.assert_array_equal(dist, want)
    bd, _ = g.sssp_batch(np.arange(16, dtype=np.uint32) + 3)
    V0 = np.full(n, INF, np.uint32)
    V0[3] = 0
    want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
    np.testing.assert_array_equal(bd[:, 0], want)


def test_selector_rejects_bad_sizes(engine):
    with pytest.raises(capi.KitesError):
        engine.selector_load(np.zeros(10, np.float32))


def test_default_selector_is_trained_and_exact(cfg1_edges):
    """A fresh engine carries the trained default selector (compiled in from
    selector_default.inc), and AUTO with it reaches the oracle's fixed point."""
    eng = capi.Engine(0)
    try:
        P = eng.selector_save()
        neutral = np.zeros(capi.SELECTOR_PARAMS, np.float32)
        neutral[capi.SEL_OFF["std"]:capi.SEL_OFF["std"] + 12] = 1.0
        assert not np.array_equal(P, neutral)
        n = 1 << 16
        s, d, w = capi.gen_rmat(16, 16 << 16, seed=8)
        R, C, E = capi.csc_from_edges(n, s, d, w)
        g = capi.Graph(eng, R, C, E)
        plain, _ = g.sssp(5)
        auto, st = g.sssp(5, opts=capi.default_opts(strategy=capi.STRATEGY_AUTO))
        np.testing.assert_array_equal(auto, plain)
        assert sum(st.strategy_hist) == st.iterations
        g.close()
    finally:
        eng.close()


def test_tpv_guard_on_hub_graph(engine):
    """Selector weights that always want the threads-per-vertex class: on an
    R-MAT graph whose hubs exceed the guard's row length, the iterations
    whose changed set holds such a row run PLAIN instead, and the result is
    the fixed point."""
    n = 1 << 18
    s, d, w = capi.gen_rmat(18, 16 * n, seed=5)
    assert np.bincount(d, minlength=n).max() >= 8192
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(engine, R, C, E)
    src = int(np.argmax(np.bincount(s, minlength=n)))   # the biggest hub changes first
    plain, _ = g.sssp(src)
    engine.selector_load(forced_selector(3))
    try:
        for loop in (0, 1):
            got, st = g.sssp(src, opts=capi.default_opts(strategy=capi.STRATEGY_AUTO,
                                                         device_loop=loop))
            np.testing.assert_array_equal(got, plain)
            assert st.strategy_hist[capi.STRATEGY_PLAIN] > 0, list(st.strategy_hist)
    finally:
        engine.selector_load(forced_selector(0))
        g.close()
