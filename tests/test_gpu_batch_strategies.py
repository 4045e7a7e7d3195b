"""Learned + batched: the batched loop's per-iteration strategies (PUSH,
PULL_ALL and PULL_CHANGED move only the changed 32-byte sectors of each
source row) and its selector reach the same V x K distances as the plain
batched pull, bit for bit, and each column equals the oracle's fixed point
for its source."""
import numpy as np
import pytest

from kites_b200 import capi
from oracle import oracle as O
from test_gpu_strategies import forced_selector

pytestmark = pytest.mark.gpu

INF = O.INF32
BATCH_STRATEGIES = [capi.STRATEGY_PUSH, capi.STRATEGY_PULL_ALL, capi.STRATEGY_PULL_CHANGED,
                    capi.STRATEGY_AUTO]


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
    engine.selector_load_batch(forced_selector(0))


def sources_for(n, k, seed):
    return np.random.default_rng(seed).choice(n, size=k, replace=False).astype(np.uint32)


@pytest.mark.parametrize("strategy", BATCH_STRATEGIES)
@pytest.mark.parametrize("k", [16, 64, 256])
@pytest.mark.parametrize("device_loop", [0, 1])
@pytest.mark.parametrize("name", [g[0] for g in GRAPHS])
def test_batched_strategy_equals_plain(uploaded, strategy, k, device_loop, name):
    g, R, C, E, n = uploaded[name]
    if k > n:
        pytest.skip("more sources than vertices")
    for op, oop in [(capi.OP_SSSP, O.OP_SSSP_SAT), (capi.OP_BFS, O.OP_BFS_SAT)]:
        srcs = sources_for(n, k, 1000 + k)
        plain, _ = g.sssp_batch(srcs, op=op, opts=capi.default_opts(device_loop=device_loop))
        got, st = g.sssp_batch(srcs, op=op, opts=capi.default_opts(strategy=strategy,
                                                                   device_loop=device_loop))
        np.testing.assert_array_equal(got, plain)
        assert sum(st.strategy_hist) == st.iterations
        j = k // 3
        V0 = np.full(n, INF, np.uint32)
        V0[srcs[j]] = 0
        want, _ = O.sanity_check(R, C, E, V0, op=oop)
        np.testing.assert_array_equal(got[:, j], want)


@pytest.mark.parametrize("cls", [0, 1, 2, 3])
@pytest.mark.parametrize("device_loop", [0, 1])
def test_batched_selector_switch_takes_each_class(engine, uploaded, cls, device_loop):
    g, R, C, E, n = uploaded["rmat14"]
    srcs = sources_for(n, 64, 7)
    plain, _ = g.sssp_batch(srcs)
    engine.selector_load_batch(forced_selector(cls))
    try:
        o = capi.default_opts(strategy=capi.STRATEGY_AUTO, device_loop=device_loop)
        got, st = g.sssp_batch(srcs, opts=o)
        np.testing.assert_array_equal(got, plain)
        assert st.strategy_hist[capi.BATCH_CLASS_STRATEGY[cls]] == st.iterations, \
            list(st.strategy_hist)
    finally:
        engine.selector_load_batch(forced_selector(0))


def test_batched_selector_mixing_classes(engine, uploaded):
    """Random weights: the selector switches classes between iterations and
    the result still equals the plain batched pull."""
    g, R, C, E, n = uploaded["rmat14"]
    srcs = sources_for(n, 64, 9)
    plain, _ = g.sssp_batch(srcs)
    rng = np.random.default_rng(5)
    try:
        mixed = 0
        for trial in range(6):
            P = forced_selector(0)
            P[capi.SEL_OFF["W1"]:] = rng.normal(0, 1.5, capi.SELECTOR_PARAMS -
                                                capi.SEL_OFF["W1"]).astype(np.float32)
            engine.selector_load_batch(P)
            got, st = g.sssp_batch(srcs, opts=capi.default_opts(strategy=capi.STRATEGY_AUTO,
                                                                selector_margin=0.0))
            np.testing.assert_array_equal(got, plain)
            mixed += sum(1 for h in st.strategy_hist if h) > 1
        assert mixed >= 1
    finally:
        engine.selector_load_batch(forced_selector(0))


def test_batched_record_fit_and_run(engine, uploaded):
    g, R, C, E, n = uploaded["rmat14"]
    X, T = [], []
    for seed in (1, 2):
        srcs = sources_for(n, 64, seed)
        x, t = g.selector_record_batch(srcs, capacity=128)
        _, st = g.sssp_batch(srcs)
        # The pulls update D in place, so a value lowered early in an
        # iteration can be read later in the same one: the iteration count
        # of two runs may differ by scheduling (the distances never do).
        assert abs(x.shape[0] - st.iterations) <= 2 and np.all(t > 0)
        X.append(x)
        T.append(t)
    single = engine.selector_save()
    params, loss = engine.selector_fit(np.concatenate(X), np.concatenate(T), epochs=300)
    assert np.isfinite(loss)
    np.testing.assert_array_equal(engine.selector_save(), single)  # fit loads nothing
    engine.selector_load_batch(params)
    np.testing.assert_array_equal(engine.selector_save_batch(), params)
    srcs = sources_for(n, 64, 3)
    plain, _ = g.sssp_batch(srcs)
    got, _ = g.sssp_batch(srcs, opts=capi.default_opts(strategy=capi.STRATEGY_AUTO,
                                                       selector_margin=0.0))
    np.testing.assert_array_equal(got, plain)
    engine.selector_load_batch(forced_selector(0))


def test_batched_strategies_reject_wrapping_and_unknown(uploaded):
    g, R, C, E, n = uploaded["rmat14"]
    srcs = sources_for(n, 16, 1)
    with pytest.raises(capi.KitesError) as e:
        g.sssp_batch(srcs, op=capi.OP_SSSP_WRAP,
                     opts=capi.default_opts(strategy=capi.STRATEGY_PUSH))
    assert e.value.status == capi.ERR_UNSUPPORTED
    with pytest.raises(capi.KitesError) as e:
        g.sssp_batch(srcs, opts=capi.default_opts(strategy=capi.STRATEGY_TPV8))
    assert e.value.status == capi.ERR_UNSUPPORTED


@pytest.mark.parametrize("strategy", [capi.STRATEGY_PULL_CHANGED])
def test_single_source_pull_changed(uploaded, strategy):
    for name in ("rmat14", "grid48"):
        g, R, C, E, n = uploaded[name]
        dist, st = g.sssp(5, opts=capi.default_opts(strategy=strategy))
        V0 = np.full(n, INF, np.uint32)
        V0[5] = 0
        want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
        np.testing.assert_array_equal(dist, want)
        assert st.strategy_hist[strategy] == st.iterations


@pytest.mark.parametrize("strategy", BATCH_STRATEGIES)
def test_batched_strategies_on_64bit_offsets(engine, uploaded, strategy):
    """The same kernels instantiated for uint64 row offsets."""
    _, R, C, E, n = uploaded["rmat14"]
    g64 = capi.Graph(engine, R, C, E, offsets64=True)
    try:
        assert g64.device_view().offsets64 == 1
        srcs = sources_for(n, 64, 21)
        plain, _ = uploaded["rmat14"][0].sssp_batch(srcs)
        got, _ = g64.sssp_batch(srcs, opts=capi.default_opts(strategy=strategy))
        np.testing.assert_array_equal(got, plain)
    finally:
        g64.close()


@pytest.mark.parametrize("strategy", [capi.STRATEGY_PLAIN, capi.STRATEGY_AUTO])
def test_async_batches_deliver_every_result(engine, uploaded, strategy):
    """kites_sssp_batch_async: three batches issued back to back, each into
    its own pinned buffer, equal the synchronous results once the engine is
    synchronised (the copies run on the second stream)."""
    import ctypes

    import torch

    g, R, C, E, n = uploaded["rmat14"]
    lib = capi.load()
    o = capi.default_opts(strategy=strategy)
    groups = [sources_for(n, 64, 40 + i) for i in range(3)]
    want = [g.sssp_batch(grp)[0] for grp in groups]
    bufs = [torch.empty((n, 64), dtype=torch.int32, pin_memory=True) for _ in groups]
    for grp, buf in zip(groups, bufs):
        capi._check(lib.kites_sssp_batch_async(engine._h, g._h, capi.OP_SSSP, capi._p(grp), 64,
                                               capi._p(buf), ctypes.byref(o), None))
    engine.sync()
    for w, buf in zip(want, bufs):
        np.testing.assert_array_equal(buf.numpy().view(np.uint32), w)
