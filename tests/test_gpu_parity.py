"""Parity of the CUDA path (through the C ABI) with the oracle and with the
golden vectors produced by the reference's own code.  Bit-exact for the
integer programs; PageRank within 1e-5 relative L1 of the FP64 oracle."""
import numpy as np
import pytest

from kites_b200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

INF = O.INF32
EX_INF = 1073741823  # the reference example's INF (sssp_basic_single_device.cu:20)


def opts(device_loop=1, **kw):
    return capi.default_opts(device_loop=device_loop, **kw)


def upload_host_graph(engine, hg):
    """Upload an oracle HostGraph the way make_graph_csr_for_device does."""
    dir_R = dir_C = None
    if hg.directed and hg.vertexPerGroup > 1:
        dir_R, dir_C = hg.dir_R, hg.dir_C
    return capi.Graph(engine, hg.R, hg.C, hg.E, V=hg.V, frontier=hg.vBitmap,
                      frontier_nbits=hg.nbits, vpg=hg.vertexPerGroup,
                      directed=hg.directed, dir_R=dir_R, dir_C=dir_C)


def cfg1_csc(cfg1_edges):
    s, d, w = cfg1_edges
    return capi.csc_from_edges(7115, s, d, w)


@pytest.mark.parametrize("device_loop", [0, 1])
def test_cfg1_sssp_golden(engine, golden, cfg1_edges, device_loop):
    R, C, E = cfg1_csc(cfg1_edges)
    g = capi.Graph(engine, R, C, E)
    for src, key in [(0, "cfg1_sssp"), (4321, "cfg1_sssp_src4321")]:
        dist, st = g.sssp(src, opts=opts(device_loop))
        np.testing.assert_array_equal(dist, golden[key][:7115])
        assert st.iterations >= 2
        assert st.edges_traversed > 0
    g.close()


def test_cfg1_bfs_golden(engine, golden, cfg1_edges):
    R, C, E = cfg1_csc(cfg1_edges)
    g = capi.Graph(engine, R, C, E)
    dist, _ = g.sssp(0, op=capi.OP_BFS)
    np.testing.assert_array_equal(dist, golden["cfg1_bfs"][:7115])


def test_cfg1_cc_golden(engine, golden, cfg1_edges):
    s, d, _ = cfg1_edges
    ss = np.concatenate([s, d])
    tt = np.concatenate([d, s])
    keys = np.unique(ss.astype(np.uint64) << np.uint64(32) | tt)
    ss = (keys >> np.uint64(32)).astype(np.uint32)
    tt = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    R, C, _ = capi.csc_from_edges(7115, ss, tt)
    g = capi.Graph(engine, R, C, None)
    labels, _ = g.cc()
    np.testing.assert_array_equal(labels, golden["cfg1_cc"][:7115])


@pytest.mark.parametrize("vpg", [1, 2, 4, 8, 16, 32, 64])
def test_reference_process_semantics_vpg(engine, cfg1_edges, vpg):
    """kites::process on a host graph built with the reference's rules
    (example pre-processing, INF 2^30-1, wrap-around add) for every vpg."""
    s, d, w = cfg1_edges
    hg = O.build_host_graph(s, d, w, vpg=vpg, init="source", source=0, inf=EX_INF)
    want, _ = O.process(hg, op=O.OP_SSSP_WRAP)
    gs, _ = O.sanity_check(hg, op=O.OP_SSSP_WRAP)
    np.testing.assert_array_equal(want, gs)
    g = upload_host_graph(engine, hg)
    st = g.process(capi.OP_SSSP_WRAP, opts())
    got = g.get_values()
    np.testing.assert_array_equal(got, want)
    assert st.iterations >= 2


def test_undirected_construction_has_empty_frontier(engine, cfg1_edges):
    """graph_csr's undirected constructor copies no frontier bits
    (graph_csr.h:100-101): process() runs one empty iteration."""
    s, d, w = cfg1_edges
    hg = O.build_host_graph(s, d, w, directed=False, incomplete=True, init="source",
                            source=0, inf=EX_INF)
    want, iters = O.process(hg, op=O.OP_SSSP_WRAP)
    np.testing.assert_array_equal(want, hg.V)
    g = upload_host_graph(engine, hg)
    st = g.process(capi.OP_SSSP_WRAP, opts())
    np.testing.assert_array_equal(g.get_values(), want)
    assert st.iterations == iters == 1


def test_undirected_with_frontier_activates_through_C(engine, cfg1_edges):
    s, d, w = cfg1_edges
    hg = O.build_host_graph(s, d, w, directed=False, incomplete=True, init="source",
                            source=0, inf=EX_INF)
    # Start from the source's neighbours, as a caller setting vBitmap would.
    bits = np.zeros(hg.n_vertices, bool)
    bits[hg.C[hg.R[0]:hg.R[1]]] = True
    hg.vBitmap = O._pack_bits(bits)
    hg.nbits = hg.n_vertices
    want, _ = O.process(hg, op=O.OP_SSSP_WRAP)
    g = upload_host_graph(engine, hg)
    g.process(capi.OP_SSSP_WRAP, opts())
    np.testing.assert_array_equal(g.get_values(), want)


def random_graph(n, m, seed, w_hi=100, dup=False, selfloops=False):
    rng = np.random.default_rng(seed)
    s = rng.integers(0, n, m, dtype=np.uint32)
    d = rng.integers(0, n, m, dtype=np.uint32)
    if not selfloops:
        keep = s != d
        s, d = s[keep], d[keep]
    if not dup:
        k = np.unique(s.astype(np.uint64) << np.uint64(32) | d)
        s = (k >> np.uint64(32)).astype(np.uint32)
        d = (k & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    w = rng.integers(1, w_hi + 1, s.shape[0], dtype=np.uint32)
    return s, d, w


@pytest.mark.parametrize("n", [1, 31, 32, 33, 127, 128, 129, 255, 1000, 4097])
@pytest.mark.parametrize("op", [capi.OP_SSSP, capi.OP_BFS])
def test_sizes_around_padding(engine, n, op):
    s, d, w = random_graph(n, 4 * n + 3, seed=n) if n > 1 else (
        np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(engine, R, C, E)
    src = n // 3
    dist, _ = g.sssp(src, op=op)
    V0 = np.full(n, INF, np.uint32)
    V0[src] = 0
    want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT if op == capi.OP_SSSP else O.OP_BFS_SAT)
    np.testing.assert_array_equal(dist, want)


def test_hub_in_and_out(engine):
    """A hub whose in- and out-rows span many chunks (atomicMin merge path)."""
    n = 50000
    rng = np.random.default_rng(7)
    others = np.arange(1, n, dtype=np.uint32)
    s = np.concatenate([others, np.zeros(n - 1, np.uint32),
                        rng.integers(0, n, 100000, dtype=np.uint32)])
    d = np.concatenate([np.zeros(n - 1, np.uint32), others,
                        rng.integers(0, n, 100000, dtype=np.uint32)])
    keep = s != d
    s, d = s[keep], d[keep]
    k = np.unique(s.astype(np.uint64) << np.uint64(32) | d)
    s = (k >> np.uint64(32)).astype(np.uint32)
    d = (k & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    w = rng.integers(1, 1000, s.shape[0], dtype=np.uint32)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(engine, R, C, E)
    for src in (0, 17, n - 1):
        dist, _ = g.sssp(src)
        V0 = np.full(n, INF, np.uint32)
        V0[src] = 0
        want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
        np.testing.assert_array_equal(dist, want)


def test_duplicates_and_selfloops(engine):
    s, d, w = random_graph(3000, 20000, seed=3, dup=True, selfloops=True)
    R, C, E = capi.csc_from_edges(3000, s, d, w)
    g = capi.Graph(engine, R, C, E)
    dist, _ = g.sssp(5)
    V0 = np.full(3000, INF, np.uint32)
    V0[5] = 0
    want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
    np.testing.assert_array_equal(dist, want)


def test_saturating_weights(engine):
    """Weights near 2^32: the built-in SSSP saturates at 0xFFFFFFFF."""
    s, d, _ = random_graph(2000, 8000, seed=11)
    rng = np.random.default_rng(11)
    w = rng.integers(0x7FFFFFFF, 0xFFFFFFFF, s.shape[0], dtype=np.uint64).astype(np.uint32)
    R, C, E = capi.csc_from_edges(2000, s, d, w)
    g = capi.Graph(engine, R, C, E)
    dist, _ = g.sssp(0)
    V0 = np.full(2000, INF, np.uint32)
    V0[0] = 0
    want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
    np.testing.assert_array_equal(dist, want)


def test_er_and_grid(engine):
    for s, d, w, n in [capi.gen_er(20000, 160000, seed=5) + (20000,),
                       capi.gen_grid(64, seed=5) + (64 * 64,)]:
        R, C, E = capi.csc_from_edges(n, s, d, w)
        g = capi.Graph(engine, R, C, E)
        dist, _ = g.sssp(1)
        V0 = np.full(n, INF, np.uint32)
        V0[1] = 0
        want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
        np.testing.assert_array_equal(dist, want)


def test_iteration_limit_times_out(engine):
    s, d, w = capi.gen_grid(32, seed=2)
    R, C, E = capi.csc_from_edges(32 * 32, s, d, w)
    g = capi.Graph(engine, R, C, E)
    for dl in (0, 1):
        with pytest.raises(capi.KitesError) as ei:
            g.sssp(0, opts=opts(dl, max_iterations=3))
        assert ei.value.status == capi.ERR_TIMEOUT
    dist, st = g.sssp(0)  # the engine stays usable
    assert st.iterations > 3


def test_pagerank_fp64_oracle(engine):
    s, d, w = capi.gen_rmat(14, 16 << 14, seed=9)
    n = 1 << 14
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(engine, R, C, E)
    pr, st = g.pagerank(n_real=n, iterations=20, damping=0.85)
    outdeg = np.bincount(s, minlength=n).astype(np.uint32)
    want = O.pagerank_f64(n, R, C, outdeg, 20, 0.85)
    rel_l1 = np.abs(pr.astype(np.float64) - want).sum() / np.abs(want).sum()
    assert rel_l1 < 1e-5, rel_l1
    assert st.iterations == 20


def test_repeated_runs_and_pool_reuse(engine, cfg1_edges):
    R, C, E = cfg1_csc(cfg1_edges)
    first = None
    for _ in range(3):
        g = capi.Graph(engine, R, C, E)
        dist, _ = g.sssp(0)
        if first is None:
            first = dist
        np.testing.assert_array_equal(dist, first)
        g.close()
    _, _, pool = engine.mem_usage()
    assert pool > 0


@pytest.mark.parametrize("k", [32, 64, 128, 256])
@pytest.mark.parametrize("device_loop", [0, 1])
def test_batch_gather_modes_agree(engine, k, device_loop):
    """TMA row gathers (gather mode 1, K >= 32) and register loads (mode 0)
    give the same V x K distances, run after run, on one graph."""
    n = 1 << 14
    s, d, w = capi.gen_rmat(14, 16 << 14, seed=31)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(engine, R, C, E)
    srcs = np.random.default_rng(100 + k).choice(n, size=k, replace=False).astype(np.uint32)
    o = capi.default_opts(device_loop=device_loop)
    g.set_batch_gather(1)
    tma, st = g.sssp_batch(srcs, opts=o)
    g.set_batch_gather(0)
    loads, _ = g.sssp_batch(srcs, opts=o)
    g.set_batch_gather(1)
    again, _ = g.sssp_batch(srcs, opts=o)
    np.testing.assert_array_equal(tma, loads)
    np.testing.assert_array_equal(again, loads)
    single, _ = g.sssp(int(srcs[k // 2]))
    np.testing.assert_array_equal(tma[:, k // 2], single)
    assert st.iterations > 1
    g.close()


@pytest.mark.parametrize("k", [16, 32, 64, 128, 256])
@pytest.mark.parametrize("strategy", [capi.STRATEGY_PLAIN, capi.STRATEGY_AUTO,
                                      capi.STRATEGY_PULL_ALL, capi.STRATEGY_PULL_CHANGED,
                                      capi.STRATEGY_PUSH])
def test_batch_async_gathers_agree(engine, k, strategy):
    """cp.async row copies into shared memory (gather mode 2) give the V x K
    distances of the register loads (mode 0), in the fixed batched loop and in
    the batched strategies' pulls (unmasked, and masked to the changed
    sectors) and masked push, and each column is the single-source result."""
    n = 1 << 14
    s, d, w = capi.gen_rmat(14, 16 << 14, seed=33)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(engine, R, C, E)
    try:
        srcs = np.random.default_rng(300 + k).choice(n, size=k, replace=False).astype(np.uint32)
        o = capi.default_opts(strategy=strategy)
        g.set_batch_gather(0)
        loads, _ = g.sssp_batch(srcs, opts=o)
        g.set_batch_gather(2)
        cpa, st = g.sssp_batch(srcs, opts=o)
        again, _ = g.sssp_batch(srcs, opts=o)
        np.testing.assert_array_equal(cpa, loads)
        np.testing.assert_array_equal(again, loads)
        for j in (0, k // 2, k - 1):
            np.testing.assert_array_equal(cpa[:, j], g.sssp(int(srcs[j]))[0])
        assert st.iterations > 1
    finally:
        g.close()


def test_batch_gather_rejects_unknown_modes(engine):
    s, d, w = capi.gen_er(1000, 4000, seed=2)
    R, C, E = capi.csc_from_edges(1000, s, d, w)
    g = capi.Graph(engine, R, C, E)
    try:
        for mode in (-1, 3):
            with pytest.raises(capi.KitesError):
                g.set_batch_gather(mode)
    finally:
        g.close()


@pytest.mark.parametrize("k", [16, 32, 64, 128, 256])
@pytest.mark.parametrize("op", [capi.OP_SSSP, capi.OP_BFS])
def test_batched_sources_match_single_source(engine, k, op):
    n = 1 << 13
    s, d, w = capi.gen_rmat(13, 16 << 13, seed=21)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(engine, R, C, E)
    rng = np.random.default_rng(k)
    srcs = rng.choice(n, size=k, replace=False).astype(np.uint32)
    dist, st = g.sssp_batch(srcs, op=op)
    assert dist.shape == (n, k)
    oop = O.OP_SSSP_SAT if op == capi.OP_SSSP else O.OP_BFS_SAT
    for j in range(0, k, max(1, k // 16)):
        V0 = np.full(n, INF, np.uint32)
        V0[srcs[j]] = 0
        want, _ = O.sanity_check(R, C, E, V0, op=oop)
        np.testing.assert_array_equal(dist[:, j], want, err_msg=f"source slot {j}")
    assert st.iterations > 1


@pytest.mark.parametrize("device_loop", [0, 1])
def test_batched_cfg1_golden_and_vpg_graph(engine, golden, cfg1_edges, device_loop):
    s, d, w = cfg1_edges
    R, C, E = capi.csc_from_edges(7115, s, d, w)
    g = capi.Graph(engine, R, C, E)
    srcs = np.array([0, 4321] + list(range(100, 114)), np.uint32)
    dist, _ = g.sssp_batch(srcs, opts=capi.default_opts(device_loop=device_loop))
    np.testing.assert_array_equal(dist[:, 0], golden["cfg1_sssp"][:7115])
    np.testing.assert_array_equal(dist[:, 1], golden["cfg1_sssp_src4321"][:7115])
    # The same through a vpg = 4 upload (vertex-level activation in batches).
    hg = O.build_host_graph(s, d, w, vpg=4, init="source", source=0, inf=INF)
    g4 = upload_host_graph(engine, hg)
    dist4, _ = g4.sssp_batch(srcs)
    # The host graph is padded to 7168 rows; the extra rows are unreachable.
    np.testing.assert_array_equal(dist4[:7115], dist)
    assert np.all(dist4[7115:] == INF)


def test_batch_rejects_bad_input(engine, cfg1_edges):
    s, d, w = cfg1_edges
    R, C, E = capi.csc_from_edges(7115, s, d, w)
    g = capi.Graph(engine, R, C, E)
    with pytest.raises(capi.KitesError) as ei:
        g.sssp_batch(np.arange(20, dtype=np.uint32))
    assert ei.value.status == capi.ERR_INVALID
    bad = np.arange(16, dtype=np.uint32)
    bad[3] = 7115
    with pytest.raises(capi.KitesError) as ei:
        g.sssp_batch(bad)
    assert ei.value.status == capi.ERR_INVALID
    dist, _ = g.sssp_batch(np.arange(16, dtype=np.uint32))  # still usable
    assert dist[0, 0] == 0


@pytest.mark.parametrize("offsets64", [0, 1])
def test_uint64_offsets_give_the_same_results(engine, offsets64):
    """Graphs past 2^32 vertices + edges keep 64-bit row offsets on the device;
    a small graph asked for that layout runs every path of the uint64
    instantiations and must agree bit for bit with the uint32 layout."""
    n = 1 << 14
    s, d, w = capi.gen_rmat(14, 16 << 14, seed=17)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g32 = capi.Graph(engine, R, C, E)
    g = capi.Graph(engine, R, C, E, offsets64=bool(offsets64))
    assert g.device_view().offsets64 == offsets64
    for strat in (capi.STRATEGY_PLAIN, capi.STRATEGY_AUTO, capi.STRATEGY_PUSH,
                  capi.STRATEGY_PULL_ALL, capi.STRATEGY_TPV8):
        o = capi.default_opts(strategy=strat)
        np.testing.assert_array_equal(g.sssp(7, opts=o)[0], g32.sssp(7)[0])
    np.testing.assert_array_equal(g.sssp(7, op=capi.OP_BFS)[0], g32.sssp(7, op=capi.OP_BFS)[0])
    srcs = np.arange(64, dtype=np.uint32) * 101
    for mode in (0, 1, 2):
        g.set_batch_gather(mode)
        np.testing.assert_array_equal(g.sssp_batch(srcs)[0], g32.sssp_batch(srcs)[0])
    g.set_batch_gather(2)
    np.testing.assert_array_equal(
        g.sssp_batch(srcs, opts=capi.default_opts(strategy=capi.STRATEGY_AUTO))[0],
        g32.sssp_batch(srcs)[0])
    pr, _ = g.pagerank(n_real=n)
    pr32, _ = g32.pagerank(n_real=n)
    assert np.abs(pr.astype(np.float64) - pr32).sum() / np.abs(pr32).sum() < 1e-6
    V0 = np.full(n, INF, np.uint32)
    V0[7] = 0
    want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
    np.testing.assert_array_equal(g.sssp(7)[0], want)
    g.close()
    g32.close()


def test_uint64_offsets_undirected_cc(engine, cfg1_edges, golden):
    s, d, _ = cfg1_edges
    ss, tt = np.concatenate([s, d]), np.concatenate([d, s])
    k = np.unique(ss.astype(np.uint64) << np.uint64(32) | tt)
    ss = (k >> np.uint64(32)).astype(np.uint32)
    tt = (k & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    R, C, _ = capi.csc_from_edges(7115, ss, tt)
    g = capi.Graph(engine, R, C, None, offsets64=True)
    labels, _ = g.cc()
    np.testing.assert_array_equal(labels, golden["cfg1_cc"][:7115])
    g.close()
