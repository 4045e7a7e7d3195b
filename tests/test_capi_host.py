"""Host-side checks of the C ABI library: it loads, exports every symbol the
header declares, its structs match the header byte for byte, its host
generators and CSC builder follow the stated rules, and bad input is an
error status.  No GPU compute calls."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from kites_b200 import capi
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "kites_b200.h")


def declared_functions():
    text = open(HEADER).read()
    decl = r"^(?:int|void|const char \*)\s*(kites_[a-z0-9_]+)\s*\("
    return sorted(set(re.findall(decl, text, re.M)))


def test_exports_every_declared_symbol():
    lib = capi.load()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(capi.EXPORTED) == names
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], check=True,
                         capture_output=True, text=True).stdout
    for name in names:
        assert re.search(rf"\bT {name}$", out, re.M), name


def test_abi_version():
    assert capi.load().kites_abi_version() == 3


def test_struct_layout_matches_header():
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "kites_b200.h"
#define P(T, f) printf(#T "." #f " %zu\n", offsetof(T, f));
int main(void) {
  printf("csc %zu\nview %zu\nopts %zu\nstats %zu\n", sizeof(kites_csc_view),
         sizeof(kites_device_view), sizeof(kites_run_opts), sizeof(kites_run_stats));
  P(kites_csc_view, on_device) P(kites_csc_view, frontier_nbits)
  P(kites_device_view, stream) P(kites_device_view, chunk_items) P(kites_run_opts, time_kernels)
  P(kites_run_stats, pull_kernel_bytes) P(kites_run_stats, iter_edges)
  P(kites_run_stats, pull_dense_bytes) P(kites_csc_view, offsets64)
  printf("tune %zu\n", sizeof(kites_tune_result));
  P(kites_tune_result, coarse_strategy) P(kites_tune_result, coarse_ms)
  printf("strategies %d\n", (int)KITES_STRATEGY_COUNT);
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as td:
        c = os.path.join(td, "l.c")
        exe = os.path.join(td, "l")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        lines = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(ln.rsplit(" ", 1) for ln in lines if ln)
    assert int(got["csc"]) == ctypes.sizeof(capi.CscView)
    assert int(got["view"]) == ctypes.sizeof(capi.DeviceView)
    assert int(got["opts"]) == ctypes.sizeof(capi.RunOpts)
    assert int(got["stats"]) == ctypes.sizeof(capi.RunStats)
    assert int(got["kites_csc_view.on_device"]) == capi.CscView.on_device.offset
    assert int(got["kites_csc_view.frontier_nbits"]) == capi.CscView.frontier_nbits.offset
    assert int(got["kites_device_view.stream"]) == capi.DeviceView.stream.offset
    assert int(got["kites_device_view.chunk_items"]) == capi.DeviceView.chunk_items.offset
    assert int(got["kites_run_opts.time_kernels"]) == capi.RunOpts.time_kernels.offset
    assert int(got["kites_run_stats.pull_kernel_bytes"]) == capi.RunStats.pull_kernel_bytes.offset
    assert int(got["kites_run_stats.iter_edges"]) == capi.RunStats.iter_edges.offset
    assert int(got["kites_run_stats.pull_dense_bytes"]) == capi.RunStats.pull_dense_bytes.offset
    assert int(got["kites_csc_view.offsets64"]) == capi.CscView.offsets64.offset
    assert int(got["tune"]) == ctypes.sizeof(capi.TuneResult)
    assert int(got["kites_tune_result.coarse_strategy"]) == capi.TuneResult.coarse_strategy.offset
    assert int(got["kites_tune_result.coarse_ms"]) == capi.TuneResult.coarse_ms.offset
    assert int(got["strategies"]) == capi.STRATEGY_COUNT


def test_default_opts():
    o = capi.default_opts()
    assert o.strategy == capi.STRATEGY_PLAIN and o.device_loop == 1
    assert o.pagerank_iterations == 20 and abs(o.damping - 0.85) < 1e-7
    assert o.selector_margin < 0   # each loop's own default margin


def test_no_device_is_an_error_not_a_fallback():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(capi.KitesError) as ei:
        capi.Engine(0)
    assert ei.value.status == capi.ERR_NO_DEVICE


def test_null_arguments_are_errors():
    lib = capi.load()
    assert lib.kites_graph_upload(None, None, None) == capi.ERR_INVALID
    assert b"null" in lib.kites_last_error_string()
    assert lib.kites_process(None, None, 0, None, None) == capi.ERR_INVALID
    assert lib.kites_engine_create(0, None) == capi.ERR_INVALID


def test_rmat_rules():
    s, d, w = capi.gen_rmat(12, 40000, seed=3, w_lo=1, w_hi=255)
    assert s.max() < 4096 and d.max() < 4096
    assert not np.any(s == d)
    keys = s.astype(np.uint64) << np.uint64(32) | d
    assert np.unique(keys).shape[0] == keys.shape[0]
    assert w.min() >= 1 and w.max() <= 255
    s2, d2, w2 = capi.gen_rmat(12, 40000, seed=3, w_lo=1, w_hi=255)
    assert np.array_equal(s, s2) and np.array_equal(d, d2) and np.array_equal(w, w2)
    # Prefix property of the top-up rule: the first k kept candidates do not
    # depend on how many edges are asked for.
    s3, d3, _ = capi.gen_rmat(12, 30000, seed=3, w_lo=1, w_hi=255)
    assert np.array_equal(s3, s[:30000]) and np.array_equal(d3, d[:30000])
    # Skew: vertex 0 is the heaviest in-degree hub of an R-MAT with a > d.
    indeg = np.bincount(d, minlength=4096)
    assert indeg[0] == indeg.max()


def test_rmat_non_power_of_two_range():
    s, d, _ = capi.gen_rmat(13, 103689, seed=1, w_lo=1, w_hi=63, n_vertices=7115)
    assert max(s.max(), d.max()) < 7115


def test_er_and_grid_rules():
    s, d, w = capi.gen_er(5000, 30000, seed=2)
    assert not np.any(s == d) and s.max() < 5000
    keys = s.astype(np.uint64) << np.uint64(32) | d
    assert np.unique(keys).shape[0] == 30000
    side = 7
    s, d, w = capi.gen_grid(side, seed=1, w_lo=1, w_hi=1000)
    assert s.shape[0] == 4 * side * (side - 1)
    r1, c1 = s // side, s % side
    r2, c2 = d // side, d % side
    assert np.all(np.abs(r1.astype(int) - r2) + np.abs(c1.astype(int) - c2) == 1)
    assert np.bincount(s, minlength=side * side).max() == 4
    assert w.min() >= 1 and w.max() <= 1000


@pytest.mark.parametrize("seed", [1, 2])
def test_csc_matches_oracle_builder(seed):
    rng = np.random.default_rng(seed)
    n = 3001
    s = rng.integers(0, n, 20000, dtype=np.uint32)
    d = rng.integers(0, n, 20000, dtype=np.uint32)
    w = rng.integers(1, 100, 20000, dtype=np.uint32)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    hg = O.build_host_graph(s, d, w)
    nn = int(max(s.max(), d.max())) + 1
    np.testing.assert_array_equal(R[: nn + 1], hg.R[: nn + 1])
    np.testing.assert_array_equal(C, hg.C)
    np.testing.assert_array_equal(E, hg.E)


def test_bad_generator_arguments():
    with pytest.raises(capi.KitesError) as ei:
        capi.gen_rmat(10, 100, a=0.9, b=0.2, c=0.1)
    assert ei.value.status == capi.ERR_INVALID
    with pytest.raises(capi.KitesError):
        capi.gen_er(1, 10)
    with pytest.raises(capi.KitesError):
        capi.csc_from_edges(10, np.array([1, 20], np.uint32), np.array([2, 3], np.uint32))
