"""Benchmark input on the CPU: the oracle's own restatement of the R-MAT
generator and CSC builder against the library's, and the binary CSC file
format written by one side and read by the other (the benchmark's reference
arm reads its graph through the oracle only, the library arm through
kites_csc_load, so both must see the same bytes)."""
import os

import numpy as np
import pytest

from kites_b200 import capi
from oracle import csc_file
from oracle import oracle as O


@pytest.mark.parametrize("scale,m,nv,seed", [(10, 5000, 0, 1), (13, 103689, 7115, 1),
                                             (16, 16 << 16, 0, 7), (12, 20000, 3000, 3)])
def test_oracle_generator_equals_library(scale, m, nv, seed):
    want = capi.gen_rmat(scale, m, seed=seed, n_vertices=nv)
    got = O.gen_rmat(scale, m, seed=seed, n_vertices=nv)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)
    n = nv or (1 << scale)
    for a, b in zip(O.csc_from_edges(n, *got), capi.csc_from_edges(n, *want)):
        np.testing.assert_array_equal(a, b)


def test_oracle_csc_keeps_parallel_edges_in_input_order():
    src = np.array([3, 1, 3, 0, 3], np.uint32)
    dst = np.array([2, 2, 2, 2, 1], np.uint32)
    w = np.array([10, 20, 30, 40, 50], np.uint32)
    R, C, E = O.csc_from_edges(4, src, dst, w)
    np.testing.assert_array_equal(R, [0, 0, 1, 5, 5])
    np.testing.assert_array_equal(C, [3, 0, 1, 3, 3])
    np.testing.assert_array_equal(E, [50, 40, 20, 10, 30])
    for a, b in zip((R, C, E), capi.csc_from_edges(4, src, dst, w)):
        np.testing.assert_array_equal(a, b)
    with pytest.raises(ValueError):
        O.csc_from_edges(3, src, dst, w)


@pytest.fixture(scope="module")
def small_csc():
    s, d, w = capi.gen_rmat(12, 40000, seed=9)
    return capi.csc_from_edges(1 << 12, s, d, w)


def test_library_file_read_by_oracle(tmp_path, small_csc):
    R, C, E = small_csc
    p = str(tmp_path / "g.csc")
    capi.csc_save(p, R, C, E, directed=True, desc="rmat scale=12 seed=9")
    R2, C2, E2, directed, desc = csc_file.read(p)
    assert directed and desc == "rmat scale=12 seed=9"
    for a, b in zip((R2, C2, E2), (R, C, E)):
        np.testing.assert_array_equal(a, b)
    assert capi.csc_info(p) == (1 << 12, C.shape[0], True, True, "rmat scale=12 seed=9")


def test_oracle_file_read_by_library(tmp_path, small_csc):
    R, C, _ = small_csc
    p = str(tmp_path / "g.csc")
    csc_file.write(p, R, C, None, directed=False, desc="unweighted")
    R2, C2, E2 = capi.csc_load(p)
    assert E2 is None
    np.testing.assert_array_equal(R2, R)
    np.testing.assert_array_equal(C2, C)
    assert capi.csc_info(p)[2:] == (False, False, "unweighted")


def test_damaged_files_are_rejected(tmp_path, small_csc):
    R, C, E = small_csc
    p = str(tmp_path / "g.csc")
    capi.csc_save(p, R, C, E)
    raw = open(p, "rb").read()
    short = str(tmp_path / "short.csc")
    open(short, "wb").write(raw[:-4])
    bad = str(tmp_path / "bad.csc")
    open(bad, "wb").write(b"NOTACSC!" + raw[8:])
    for q in (short, bad, str(tmp_path / "missing.csc")):
        with pytest.raises(capi.KitesError):
            capi.csc_load(q)
        with pytest.raises((ValueError, OSError)):
            csc_file.read(q)
    assert not [f for f in os.listdir(tmp_path) if ".tmp" in f]


def test_save_rejects_inconsistent_offsets(tmp_path, small_csc):
    R, C, E = small_csc
    with pytest.raises(capi.KitesError):
        capi.csc_save(str(tmp_path / "g.csc"), R, C[:-1], E[:-1])


def test_reference_loop_on_many_threads(has_reference, small_csc):
    """The threaded entry of the reference harness (the benchmark's reference
    arm) gives each source the oracle's fixed point and its reached edges."""
    import bench
    lib = bench.load_ref_lib()
    if lib is None:
        pytest.skip("reference harness not built")
    R, C, E = small_csc
    n = R.shape[0] - 1
    outdeg = np.bincount(C, minlength=n).astype(np.uint64)
    srcs = bench.pick_sources(outdeg, 6, seed=2)
    secs, reached, dist = bench.time_reference(lib, n, C.shape[0], R.astype(np.uint32), C, E,
                                               outdeg, srcs, threads=3, want_dist=True)
    assert secs > 0
    for j, s in enumerate(srcs):
        V0 = np.full(n, O.INF32, np.uint32)
        V0[s] = 0
        want, _ = O.sanity_check(R, C, E, V0, op=O.OP_SSSP_SAT)
        np.testing.assert_array_equal(dist[j], want)
        assert reached[j] == bench.reached_edges(want, outdeg)
