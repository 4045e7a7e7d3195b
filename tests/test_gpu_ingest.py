"""kites_graph_from_edges: the CSC built on the device must equal the host
construction (csc_from_edges, the reference's graph_raw.h:57-190 order:
rows by destination, sources ascending, parallel edges in input order)
array for array, and runs on it must give the same answers."""
import numpy as np
import pytest

from kites_b200 import capi

pytestmark = pytest.mark.gpu


def dev_array(ptr, n, typestr):
    import torch

    class _View:
        pass

    v = _View()
    v.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr,
                                  "data": (int(ptr), False), "version": 3}
    return torch.as_tensor(v, device="cuda").cpu().numpy()


def csc_of(g):
    dv = g.device_view()
    n1 = int(dv.n_vertices) + 1
    R = dev_array(dv.R, n1, "<i8" if dv.offsets64 else "<i4").view(
        np.uint64 if dv.offsets64 else np.uint32).astype(np.uint64)
    C = dev_array(dv.C, dv.n_edges, "<i4").view(np.uint32)
    E = dev_array(dv.E, dv.n_edges, "<i4").view(np.uint32) if dv.E else None
    return R, C, E


def test_device_build_matches_host_build(engine):
    n = 1 << 14
    s, d, w = capi.gen_rmat(14, 16 * n, seed=21, w_lo=1, w_hi=255)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    host = capi.Graph(engine, R, C, E)
    dev = capi.Graph.from_edges(engine, n, s, d, w)
    for a, b in zip(csc_of(host), csc_of(dev)):
        np.testing.assert_array_equal(a, b)
    for src in (0, 77, 5000):
        np.testing.assert_array_equal(host.sssp(src)[0], dev.sssp(src)[0])
    host.close()
    dev.close()


def test_parallel_edges_keep_input_order(engine):
    rng = np.random.default_rng(5)
    n = 3000
    s = rng.integers(0, n, 40000, dtype=np.uint32)
    d = rng.integers(0, n, 40000, dtype=np.uint32)
    s[20000:] = s[:20000]  # every pair twice, with other weights
    d[20000:] = d[:20000]
    w = rng.integers(1, 1000, 40000, dtype=np.uint32)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    dev = capi.Graph.from_edges(engine, n, s, d, w)
    Rd, Cd, Ed = csc_of(dev)
    np.testing.assert_array_equal(Rd[: n + 1], R.astype(np.uint64))
    np.testing.assert_array_equal(Cd, C)
    np.testing.assert_array_equal(Ed, E)
    dev.close()


def test_device_build_from_device_pointers_unweighted(engine):
    import torch

    n = 1 << 12
    s, d, _ = capi.gen_rmat(12, 8 * n, seed=3)
    R, C, _ = capi.csc_from_edges(n, s, d, None)
    ts = torch.from_numpy(s.view(np.int32)).cuda()
    td = torch.from_numpy(d.view(np.int32)).cuda()
    dev = capi.Graph.from_edges(engine, n, ts, td, None)
    Rd, Cd, Ed = csc_of(dev)
    assert Ed is None
    np.testing.assert_array_equal(Cd, C)
    np.testing.assert_array_equal(Rd[: n + 1], R.astype(np.uint64))
    lv, _ = dev.sssp(1, op=capi.OP_BFS)
    host = capi.Graph(engine, R, C)
    np.testing.assert_array_equal(lv, host.sssp(1, op=capi.OP_BFS)[0])
    dev.close()
    host.close()


def test_device_build_rejects_bad_endpoint(engine):
    s = np.array([0, 1, 2], np.uint32)
    d = np.array([1, 2, 9], np.uint32)
    with pytest.raises(capi.KitesError) as e:
        capi.Graph.from_edges(engine, 5, s, d)
    assert e.value.status == capi.ERR_INVALID
