"""The oracle itself, pinned against the reference's own code (golden vectors
from oracle/_ref/ref_harness, and the live harness when the reference tree
is present).  CPU only."""
import hashlib
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import oracle as O

EX_INF = 1073741823
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def struct_hash(hg):
    h = hashlib.sha256()
    for a in (hg.R.astype(np.uint32), hg.C, hg.E, hg.V, hg.vBitmap,
              hg.dir_R.astype(np.uint32), hg.dir_C):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.digest()


def edges_hash(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.digest()


def test_generator_pinned(golden, cfg1_edges):
    assert edges_hash(*cfg1_edges) == bytes(golden["cfg1_edges_sha"])


@pytest.mark.parametrize("vpg", [1, 2, 4, 8])
def test_builder_matches_reference_cfg1(golden, cfg1_edges, vpg):
    s, d, w = cfg1_edges
    hg = O.build_host_graph(s, d, w, vpg=vpg, init="source", source=0, inf=EX_INF)
    assert struct_hash(hg) == bytes(golden[f"cfg1_struct_vpg{vpg}"])


@pytest.mark.parametrize("vpg", [1, 2, 4, 8, 32, 64])
def test_builder_matches_reference_wiki(golden, has_reference, vpg):
    if not has_reference:
        pytest.skip("reference example file not present")
    from conftest import WIKI
    a, b, w = O.read_edge_list(WIKI)
    hg = O.build_host_graph(a, b, w, vpg=vpg, init="source", source=30, inf=EX_INF,
                            weight_rule=O.example_weight_rule)
    assert struct_hash(hg) == bytes(golden[f"wiki_struct_vpg{vpg}"])


def mipmap_hash(hg, cr):
    dim, bits, mip = O.mipmap_of(hg, cr)
    return dim, edges_hash(hg.V, hg.R.astype(np.uint32), hg.C, hg.E, bits, mip)


@pytest.mark.parametrize("cr", [1, 3, 32, 100])
def test_mipmap_matches_reference_cfg1(golden, cfg1_edges, cr):
    """kites::graph_csr_mipmapped's block frontier and mipmap, from the
    reference's own class (graph_csr_mipmapped.hpp:40-78)."""
    s, d, w = cfg1_edges
    hg = O.build_host_graph(s, d, w, init="source", source=0, inf=EX_INF)
    dim, h = mipmap_hash(hg, cr)
    assert dim == golden["meta"]["cfg1_mipmap_dim"][str(cr)]
    assert h == bytes(golden[f"cfg1_mipmap_cr{cr}"])


@pytest.mark.parametrize("cr", [1, 3, 32, 100, 1000])
def test_mipmap_from_edges_matches_class(cfg1_edges, cr):
    """The edge-list form the engine's block map is checked against equals the
    class form over the padded vertex count."""
    s, d, w = cfg1_edges
    hg = O.build_host_graph(s, d, w, init="source", source=0, inf=EX_INF)
    dim, _, mip = O.mipmap_of(hg, cr)
    dim2, mip2 = O.mipmap_from_edges(hg.n_vertices, s, d, cr)
    assert hg.n_vertices == 7168 and dim == dim2
    np.testing.assert_array_equal(mip, mip2)


@pytest.mark.parametrize("cr", [1, 3, 32, 100])
def test_mipmap_matches_reference_wiki(golden, has_reference, cr):
    if not has_reference:
        pytest.skip("reference example file not present")
    from conftest import WIKI
    a, b, w = O.read_edge_list(WIKI)
    hg = O.build_host_graph(a, b, w, init="source", source=30, inf=EX_INF,
                            weight_rule=O.example_weight_rule)
    dim, h = mipmap_hash(hg, cr)
    assert dim == golden["meta"]["wiki"]["mipmap_dim"][str(cr)]
    assert h == bytes(golden[f"wiki_mipmap_cr{cr}"])


def test_wiki_fixed_point_and_process(golden, has_reference):
    if not has_reference:
        pytest.skip("reference example file not present")
    from conftest import WIKI
    a, b, w = O.read_edge_list(WIKI)
    hg = O.build_host_graph(a, b, w, init="source", source=30, inf=EX_INF,
                            weight_rule=O.example_weight_rule)
    V, sweeps = O.sanity_check(hg, op=O.OP_SSSP_WRAP)
    np.testing.assert_array_equal(V, golden["wiki_sssp"])
    assert sweeps == golden["meta"]["wiki"]["sweeps"]
    Vp, _ = O.process(hg, op=O.OP_SSSP_WRAP)
    np.testing.assert_array_equal(Vp, golden["wiki_sssp"])


def test_wiki_undirected_construction(golden, has_reference):
    if not has_reference:
        pytest.skip("reference example file not present")
    from conftest import WIKI
    a, b, w = O.read_edge_list(WIKI)
    hg = O.build_host_graph(a, b, w, directed=False, incomplete=True, init="source",
                            source=30, inf=EX_INF, weight_rule=O.example_weight_rule)
    assert struct_hash(hg) == bytes(golden["wiki_undir_struct"])
    assert not hg.vBitmap.any()           # no frontier bits copied
    V, _ = O.sanity_check(hg, op=O.OP_SSSP_WRAP)
    np.testing.assert_array_equal(V, golden["wiki_undir_fix"])
    Vp, iters = O.process(hg, op=O.OP_SSSP_WRAP)
    np.testing.assert_array_equal(Vp, hg.V)  # process() changes nothing
    assert iters == 1


def cfg1_graph(cfg1_edges):
    s, d, w = cfg1_edges
    return O.build_host_graph(s, d, w, init="source", source=0, inf=O.INF32)


def test_cfg1_golden_fixed_points(golden, cfg1_edges):
    hg = cfg1_graph(cfg1_edges)
    for src, key in [(0, "cfg1_sssp"), (4321, "cfg1_sssp_src4321")]:
        V0 = np.full(hg.n_vertices, O.INF32, np.uint32)
        V0[src] = 0
        V, _ = O.sanity_check(hg.R, hg.C, hg.E, V0, op=O.OP_SSSP_SAT)
        np.testing.assert_array_equal(V, golden[key])
        ok, msg = O.certify_shortest_paths(hg.R, hg.C, hg.E, V, [src])
        assert ok, msg
    V0 = np.full(hg.n_vertices, O.INF32, np.uint32)
    V0[0] = 0
    Vb, _ = O.sanity_check(hg.R, hg.C, None, V0, op=O.OP_BFS_SAT)
    np.testing.assert_array_equal(Vb, golden["cfg1_bfs"])
    ok, msg = O.certify_shortest_paths(hg.R, hg.C, hg.E, Vb, [0], unit_weight=True)
    assert ok, msg


def test_cfg1_cc_golden(golden, cfg1_edges):
    s, d, _ = cfg1_edges
    ss, tt = np.concatenate([s, d]), np.concatenate([d, s])
    k = np.unique(ss.astype(np.uint64) << np.uint64(32) | tt)
    ss = (k >> np.uint64(32)).astype(np.uint32)
    tt = (k & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    hs = O.build_host_graph(ss, tt, None, init="label")
    L, _ = O.sanity_check(hs.R, hs.C, None, np.arange(hs.n_vertices, dtype=np.uint32),
                          op=O.OP_CC_MIN)
    np.testing.assert_array_equal(L, golden["cfg1_cc"])
    ok, msg = O.certify_min_label(hs.R, hs.C, L)
    assert ok, msg


def random_hg(n, m, seed, vpg=1, init="source", source=0):
    rng = np.random.default_rng(seed)
    s = rng.integers(0, n, m, dtype=np.uint32)
    d = rng.integers(0, n, m, dtype=np.uint32)
    w = rng.integers(1, 60, m, dtype=np.uint32)
    return O.build_host_graph(s, d, w, vpg=vpg, init=init, source=source, inf=EX_INF)


@pytest.mark.parametrize("vpg", [1, 2, 4, 16, 32, 128])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_process_equals_gauss_seidel(vpg, seed):
    hg = random_hg(700, 3000, seed, vpg=vpg, source=seed)
    gs, _ = O.sanity_check(hg, op=O.OP_SSSP_WRAP)
    pr, _ = O.process(hg, op=O.OP_SSSP_WRAP)
    np.testing.assert_array_equal(pr, gs)
    ja, _ = O.jacobi_fixed_point(hg.R, hg.C, hg.E, hg.V, op=O.OP_SSSP_WRAP)
    np.testing.assert_array_equal(ja, gs)


def test_certificate_rejects_planted_mistakes(cfg1_edges):
    hg = cfg1_graph(cfg1_edges)
    V0 = np.full(hg.n_vertices, O.INF32, np.uint32)
    V0[0] = 0
    V, _ = O.sanity_check(hg.R, hg.C, hg.E, V0, op=O.OP_SSSP_SAT)
    reached = np.flatnonzero((V != O.INF32) & (V > 0))
    bad = V.copy()
    bad[reached[5]] += 1                       # too long: a tight edge relaxes it
    assert not O.certify_shortest_paths(hg.R, hg.C, hg.E, bad, [0])[0]
    bad = V.copy()
    bad[reached[7]] -= 1                       # too short: no tight in-edge
    assert not O.certify_shortest_paths(hg.R, hg.C, hg.E, bad, [0])[0]
    bad = V.copy()
    bad[0] = 3
    assert not O.certify_shortest_paths(hg.R, hg.C, hg.E, bad, [0])[0]


def test_pagerank_oracle_dense_small():
    rng = np.random.default_rng(4)
    n = 50
    s = rng.integers(0, n, 300, dtype=np.uint32)
    d = rng.integers(0, n, 300, dtype=np.uint32)
    hg = O.build_host_graph(s, d, None, init="label")
    outdeg = np.bincount(s, minlength=n).astype(np.uint32)
    pr = O.pagerank_f64(n, hg.R, hg.C, outdeg, 20, 0.85)
    M = np.zeros((n, n))
    for a, b in zip(s.tolist(), d.tolist()):
        M[b, a] += 1.0 / outdeg[a]
    x = np.full(n, 1.0 / n)
    for _ in range(20):
        x = 0.15 / n + 0.85 * M @ x
    np.testing.assert_allclose(pr, x, rtol=1e-12, atol=1e-15)


def _harness_csc(R, C, E, V, op):
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "i"), os.path.join(td, "o")
        with open(inp, "wb") as f:
            f.write(np.array([V.shape[0], C.shape[0]], np.uint64).tobytes())
            f.write(V.tobytes())
            f.write(R.astype(np.uint32).tobytes())
            f.write(C.tobytes())
            f.write(E.tobytes())
        subprocess.run([HARNESS, "csc", inp, op, out], check=True, capture_output=True)
        with open(out, "rb") as f:
            f.read(8)
            return np.frombuffer(f.read(), np.uint32)


@pytest.mark.parametrize("seed", [11, 12, 13, 14])
def test_live_reference_harness(has_reference, seed):
    if not (has_reference and os.path.exists(HARNESS)):
        pytest.skip("reference harness not built")
    hg = random_hg(2000, 9000, seed)
    V0 = np.full(hg.n_vertices, O.INF32, np.uint32)
    V0[seed] = 0
    for op_name, op in [("sssp_sat", O.OP_SSSP_SAT), ("bfs", O.OP_BFS_SAT)]:
        want = _harness_csc(hg.R, hg.C, hg.E, V0, op_name)
        got, _ = O.sanity_check(hg.R, hg.C, hg.E, V0, op=op)
        np.testing.assert_array_equal(got, want)
    L0 = np.arange(hg.n_vertices, dtype=np.uint32)
    np.testing.assert_array_equal(O.sanity_check(hg.R, hg.C, hg.E, L0, op=O.OP_CC_MIN)[0],
                                  _harness_csc(hg.R, hg.C, hg.E, L0, "cc"))


def test_union_find_labels_equal_reference_cc(golden, cfg1_edges):
    """The exact min-label oracle used at full size equals the reference's
    own CC fixed point on config 1's symmetrised graph."""
    s, d, _ = cfg1_edges
    lab = O.cc_min_labels(7115, s, d)
    want = golden["cfg1_cc"][:7115]
    touched = np.zeros(7115, bool)
    touched[s] = touched[d] = True
    np.testing.assert_array_equal(lab[touched], want[touched])


def test_union_find_labels_equal_min_label_sweep():
    from kites_b200 import capi
    for seed in (1, 2, 3):
        s, d, _ = capi.gen_er(3000, 2000, seed=seed)
        lab = O.cc_min_labels(3000, s, d)
        R, C, _ = capi.csc_from_edges(3000, np.concatenate([s, d]), np.concatenate([d, s]))
        want, _ = O.sanity_check(R, C, None, np.arange(3000, dtype=np.uint32), op=O.OP_CC_MIN)
        np.testing.assert_array_equal(lab, want)
