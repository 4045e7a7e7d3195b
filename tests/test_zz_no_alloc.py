"""kites_sssp_noalloc: the shortest-path entry point for callers that cannot
allocate device memory when they need the answer (memory reserved up front
with allocation forbidden on the serving path, or device memory owned by
another runtime's allocator).  The caller passes buffers it already owns;
the entry point's scratch is a fixed array compiled into the library.

Its output must equal the allocating entry point's (kites_sssp) bit for bit,
on two calls in a row -- the calls share that fixed array, so the second
one also checks that the first one's leftovers are cleared.  This file is
collected last on purpose."""
import ctypes

import numpy as np
import pytest

from kites_b200 import capi

pytestmark = pytest.mark.gpu


def call_noalloc(dv, n, m, source, dist_ptr):
    it = ctypes.c_uint32()
    st = capi.load().kites_sssp_noalloc(dv.R, dv.C, dv.E, m, dv.dir_R, dv.dir_C, n, source,
                                        dist_ptr, None, ctypes.byref(it))
    return st, it.value


def test_noalloc_matches_allocating_entry_point(engine):
    import torch

    n = 1 << 15
    s, d, w = capi.gen_rmat(15, 16 << 15, seed=77, w_lo=1, w_hi=255)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(engine, R, C, E)
    dv = g.device_view()
    assert dv.offsets64 == 0 and dv.n_vertices == n
    m = int(C.shape[0])
    dist = torch.empty(n, dtype=torch.int32, device="cuda")
    for source in (11, 4242):  # two calls in a row on the shared scratch
        st, iters = call_noalloc(dv, n, m, source, dist.data_ptr())
        assert st == capi.OK, capi.load().kites_last_error_string()
        assert iters >= 2
        torch.cuda.synchronize()
        got = dist.cpu().numpy().view(np.uint32)
        want, _ = g.sssp(source)
        np.testing.assert_array_equal(got, want)
    g.close()


def test_noalloc_rejects_sizes_beyond_its_scratch(engine):
    lib = capi.load()
    one = ctypes.c_void_p(1)  # never dereferenced: the size check comes first
    st = lib.kites_sssp_noalloc(one, one, one, 0, one, one, (1 << 24) + 1, 0, one, None, None)
    assert st == capi.ERR_INVALID
    assert b"16777216" in lib.kites_last_error_string()
