"""ctypes binding of include/kites_b200.h (libkites_b200.so, built in-tree).

This is how Python callers -- the parity tests, bench.py, smoke() -- reach
the engine: through the same C ABI the C++ front-end in include/kites/
uses.  There is no fallback: if the shared library is missing,
``load()`` raises.
"""
from __future__ import annotations

import ctypes
import os
import weakref
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int,
                    c_int32, c_uint8, c_uint32, c_uint64, c_void_p)

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkites_b200.so")

OK, ERR_INVALID, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_NO_DEVICE = range(7)
OP_SSSP, OP_SSSP_WRAP, OP_BFS, OP_CC, OP_PAGERANK = range(5)
(STRATEGY_PLAIN, STRATEGY_AUTO, STRATEGY_PUSH, STRATEGY_PULL_ALL, STRATEGY_TPV1,
 STRATEGY_TPV4, STRATEGY_TPV8, STRATEGY_TPV32, STRATEGY_PULL_CHANGED, STRATEGY_MIP) = range(10)
STRATEGY_COUNT = 10
MAX_RECORDED_ITERS = 4096
INF = 0xFFFFFFFF

# Every symbol include/kites_b200.h declares.
EXPORTED = [
    "kites_last_error_string", "kites_abi_version", "kites_default_run_opts",
    "kites_engine_create", "kites_engine_destroy", "kites_engine_mem_usage",
    "kites_engine_sync", "kites_engine_stream", "kites_graph_upload", "kites_graph_destroy",
    "kites_graph_device_view", "kites_graph_get_values", "kites_graph_set_values",
    "kites_graph_set_frontier", "kites_process", "kites_sssp", "kites_sssp_batch",
    "kites_cc", "kites_pagerank", "kites_gen_rmat", "kites_gen_er", "kites_gen_grid",
    "kites_csc_from_edges", "kites_selector_record", "kites_selector_train",
    "kites_selector_load", "kites_selector_save", "kites_graph_set_tpv",
    "kites_sssp_multi_seed", "kites_gen_rmat_union", "kites_autotune",
    "kites_graph_set_density", "kites_sssp_noalloc", "kites_graph_from_edges",
    "kites_graph_set_batch_gather", "kites_csc_save", "kites_csc_info", "kites_csc_load",
    "kites_selector_fit", "kites_selector_record_batch", "kites_selector_load_batch",
    "kites_selector_save_batch", "kites_graph_activate", "kites_sssp_batch_async",
    "kites_engine_join", "kites_graph_build_mipmap", "kites_graph_get_mipmap",
    "kites_graph_set_coarse",
]
# Selector classes of the batched loop (kites_sssp_batch with AUTO).
BATCH_CLASS_STRATEGY = [STRATEGY_PLAIN, STRATEGY_PUSH, STRATEGY_PULL_ALL, STRATEGY_PULL_CHANGED]
SELECTOR_FEATURES, SELECTOR_CLASSES, SELECTOR_PARAMS = 12, 4, 1628
# Parameter layout of the selector MLP (offsets into the 1628 floats).
SEL_OFF = {"mean": 0, "std": 12, "W1": 24, "b1": 408, "W2": 440, "b2": 1464, "W3": 1496,
           "b3": 1624}
# Class 2 is the graph's coarse class (PULL_ALL unless set to MIP), class 3
# its threads-per-vertex width.
CLASS_STRATEGY = [STRATEGY_PLAIN, STRATEGY_PUSH, STRATEGY_PULL_ALL, None]  # None: graph's TPV


class CscView(Structure):
    _fields_ = [
        ("n_vertices", c_uint64), ("n_edges", c_uint64),
        ("row_offsets", c_void_p), ("row_offsets32", c_void_p),
        ("col_indices", c_void_p), ("edge_values", c_void_p),
        ("edge_value_size", c_uint32), ("vertex_value_size", c_uint32),
        ("vertex_values", c_void_p), ("vertex_per_group", c_uint32),
        ("directed", c_int32), ("frontier_bits", c_void_p),
        ("frontier_nbits", c_uint64), ("n_out_rows", c_uint64),
        ("out_row_offsets", c_void_p), ("out_row_offsets32", c_void_p),
        ("out_col_indices", c_void_p), ("n_out_edges", c_uint64),
        ("on_device", c_int32), ("offsets64", c_int32),
    ]


class DeviceView(Structure):
    _fields_ = [
        ("n_vertices", c_uint64), ("n_edges", c_uint64), ("nbits", c_uint64),
        ("vertex_per_group", c_uint32), ("directed", c_int32), ("offsets64", c_int32),
        ("V", c_void_p), ("R", c_void_p), ("C", c_void_p), ("E", c_void_p),
        ("dir_R", c_void_p), ("dir_C", c_void_p), ("frontier", c_void_p * 2),
        ("update_flag", c_void_p), ("stream", c_void_p), ("changed", c_void_p * 2),
        ("chunk_rows", c_void_p), ("n_chunks", c_uint64), ("chunk_items", c_uint32),
    ]


class RunOpts(Structure):
    _fields_ = [
        ("strategy", c_int32), ("device_loop", c_int32),
        ("max_iterations", c_uint64), ("pagerank_iterations", c_uint32),
        ("damping", c_float), ("selector_margin", c_float),
        ("record_iterations", c_int32), ("time_kernels", c_int32),
    ]


class RunStats(Structure):
    _fields_ = [
        ("iterations", c_uint64), ("device_ms", c_double), ("host_ms", c_double),
        ("edges_traversed", c_uint64), ("algorithmic_bytes", c_uint64),
        ("strategy_hist", c_uint64 * STRATEGY_COUNT), ("kernel_launches", c_uint64),
        ("pull_kernel_ms", c_double), ("pull_kernel_launches", c_uint64),
        ("pull_kernel_bytes", c_uint64),
        ("n_recorded", c_uint32),
        ("iter_strategy", c_uint8 * MAX_RECORDED_ITERS),
        ("iter_ms", c_float * MAX_RECORDED_ITERS),
        ("iter_active", c_uint64 * MAX_RECORDED_ITERS),
        ("iter_edges", c_uint64 * MAX_RECORDED_ITERS),
        ("pull_dense_ms", c_double), ("pull_dense_launches", c_uint64),
        ("pull_dense_bytes", c_uint64),
    ]


class TuneResult(Structure):
    _fields_ = [
        ("batch_chunk_items", c_uint32), ("tpv_strategy", c_int32),
        ("dense_edges", c_uint64), ("dense_rows", c_uint64), ("batch_ms", c_float),
        ("plain_ms", c_float), ("tpv_ms", c_float), ("trials", c_uint32),
        ("coarse_strategy", c_int32), ("coarse_ms", c_float),
    ]


class KitesError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"kites status {status}: {msg}")
        self.status = status


_lib = None


def load(path: str = LIB_PATH):
    """Load the in-tree shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing; run `python -m kites_b200.build`")
    lib = ctypes.CDLL(path)
    vp, u32, u64 = c_void_p, c_uint32, c_uint64
    sigs = {
        "kites_last_error_string": (c_char_p, []),
        "kites_abi_version": (c_int, []),
        "kites_default_run_opts": (None, [POINTER(RunOpts)]),
        "kites_engine_create": (c_int, [c_int, POINTER(c_void_p)]),
        "kites_engine_destroy": (c_int, [vp]),
        "kites_engine_mem_usage": (c_int, [vp, POINTER(c_uint64), POINTER(c_uint64),
                                           POINTER(c_uint64)]),
        "kites_engine_sync": (c_int, [vp]),
        "kites_engine_stream": (c_int, [vp, POINTER(c_void_p)]),
        "kites_graph_upload": (c_int, [vp, POINTER(CscView), POINTER(c_void_p)]),
        "kites_graph_destroy": (c_int, [vp]),
        "kites_graph_device_view": (c_int, [vp, POINTER(DeviceView)]),
        "kites_graph_get_values": (c_int, [vp, vp, u64]),
        "kites_graph_set_values": (c_int, [vp, vp, u64]),
        "kites_graph_set_frontier": (c_int, [vp, vp, u64]),
        "kites_process": (c_int, [vp, vp, c_int, POINTER(RunOpts), POINTER(RunStats)]),
        "kites_sssp": (c_int, [vp, vp, c_int, u32, vp, POINTER(RunOpts),
                               POINTER(RunStats)]),
        "kites_sssp_batch": (c_int, [vp, vp, c_int, vp, u32, vp, POINTER(RunOpts),
                                     POINTER(RunStats)]),
        "kites_cc": (c_int, [vp, vp, vp, POINTER(RunOpts), POINTER(RunStats)]),
        "kites_pagerank": (c_int, [vp, vp, u64, vp, POINTER(RunOpts), POINTER(RunStats)]),
        "kites_gen_rmat": (c_int, [u32, u64, u64, c_double, c_double, c_double, u64,
                                   u32, u32, vp, vp, vp]),
        "kites_gen_er": (c_int, [u64, u64, u64, u32, u32, vp, vp, vp]),
        "kites_gen_grid": (c_int, [u32, u64, u32, u32, vp, vp, vp]),
        "kites_csc_from_edges": (c_int, [u64, u64, vp, vp, vp, vp, vp, vp]),
        "kites_selector_record": (c_int, [vp, vp, c_int, u32, vp, vp, u32, POINTER(c_uint32)]),
        "kites_selector_train": (c_int, [vp, vp, vp, u32, u32, c_float, u64, vp,
                                         POINTER(c_float)]),
        "kites_selector_load": (c_int, [vp, vp, u32]),
        "kites_selector_save": (c_int, [vp, vp, u32]),
        "kites_graph_set_tpv": (c_int, [vp, c_int]),
        "kites_sssp_multi_seed": (c_int, [vp, vp, c_int, vp, u64, vp, POINTER(RunOpts),
                                          POINTER(RunStats)]),
        "kites_gen_rmat_union": (c_int, [u32, u64, u32, u32, u32, u32, u32, u32, vp, vp, vp,
                                         vp, vp]),
        "kites_autotune": (c_int, [vp, vp, c_int, vp, u32, u32, POINTER(TuneResult)]),
        "kites_graph_set_density": (c_int, [vp, u64, u64]),
        "kites_sssp_noalloc": (c_int, [vp, vp, vp, u64, vp, vp, u32, u32, vp, vp,
                                       POINTER(c_uint32)]),
        "kites_graph_from_edges": (c_int, [vp, u64, u64, vp, vp, vp, c_int, vp]),
        "kites_graph_set_batch_gather": (c_int, [vp, c_int]),
        "kites_csc_save": (c_int, [c_char_p, u64, u64, vp, vp, vp, c_int, c_char_p]),
        "kites_csc_info": (c_int, [c_char_p, POINTER(c_uint64), POINTER(c_uint64),
                                   POINTER(c_int), POINTER(c_int), c_char_p, ctypes.c_size_t]),
        "kites_csc_load": (c_int, [c_char_p, vp, vp, vp]),
        "kites_selector_fit": (c_int, [vp, vp, vp, u32, u32, c_float, u64, vp,
                                       POINTER(c_float)]),
        "kites_selector_record_batch": (c_int, [vp, vp, c_int, vp, u32, vp, vp, u32,
                                                POINTER(c_uint32)]),
        "kites_selector_load_batch": (c_int, [vp, vp, u32]),
        "kites_selector_save_batch": (c_int, [vp, vp, u32]),
        "kites_graph_activate": (c_int, [vp, vp, vp]),
        "kites_sssp_batch_async": (c_int, [vp, vp, c_int, vp, u32, vp, POINTER(RunOpts),
                                           POINTER(RunStats)]),
        "kites_engine_join": (c_int, [vp]),
        "kites_graph_build_mipmap": (c_int, [vp, u64]),
        "kites_graph_get_mipmap": (c_int, [vp, POINTER(c_uint64), vp, u64]),
        "kites_graph_set_coarse": (c_int, [vp, c_int]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(status):
    if status != OK:
        msg = load().kites_last_error_string().decode(errors="replace")
        raise KitesError(status, msg)


def _p(a):
    """Pointer of a numpy array, a torch tensor, or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(c_void_p)
    if hasattr(a, "data_ptr"):
        return c_void_p(a.data_ptr())
    if isinstance(a, int):
        return c_void_p(a)
    raise TypeError(type(a))


def default_opts(**kw) -> RunOpts:
    o = RunOpts()
    load().kites_default_run_opts(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


# ---------------------------------------------------------------------------
# Objects
# ---------------------------------------------------------------------------

class Engine:
    """One GPU (the reference's kites::nv_gpu, kites/device/nv_gpu.cuh:21-88)."""

    def __init__(self, device: int = 0):
        self._h = c_void_p()
        self._graphs = weakref.WeakSet()
        _check(load().kites_engine_create(device, ctypes.byref(self._h)))
        self.device = device

    def close(self):
        # The C engine destroys its graphs with it; close the Python handles
        # first so none of them is destroyed twice.
        for g in list(self._graphs):
            g.close()
        if self._h:
            load().kites_engine_destroy(self._h)
            self._h = c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def mem_usage(self):
        used, total, pool = c_uint64(), c_uint64(), c_uint64()
        _check(load().kites_engine_mem_usage(self._h, ctypes.byref(used),
                                             ctypes.byref(total), ctypes.byref(pool)))
        return used.value, total.value, pool.value

    def sync(self):
        _check(load().kites_engine_sync(self._h))

    # ---- learned selector ----
    def selector_train(self, features, times_ms, epochs=2000, lr=3e-3, seed=1):
        X = np.ascontiguousarray(features, dtype=np.float32)
        T = np.ascontiguousarray(times_ms, dtype=np.float32)
        params = np.empty(SELECTOR_PARAMS, dtype=np.float32)
        loss = c_float()
        _check(load().kites_selector_train(self._h, _p(X), _p(T), X.shape[0], epochs, lr,
                                           seed, _p(params), ctypes.byref(loss)))
        return params, loss.value

    def selector_load(self, params):
        P = np.ascontiguousarray(params, dtype=np.float32)
        _check(load().kites_selector_load(self._h, _p(P), P.shape[0]))

    def selector_save(self):
        P = np.empty(SELECTOR_PARAMS, dtype=np.float32)
        _check(load().kites_selector_save(self._h, _p(P), SELECTOR_PARAMS))
        return P

    def selector_fit(self, features, times_ms, epochs=2000, lr=3e-3, seed=1):
        """Fits the MLP to recorded timings; returns (params, loss), loads nothing."""
        X = np.ascontiguousarray(features, dtype=np.float32)
        T = np.ascontiguousarray(times_ms, dtype=np.float32)
        params = np.empty(SELECTOR_PARAMS, dtype=np.float32)
        loss = c_float()
        _check(load().kites_selector_fit(self._h, _p(X), _p(T), X.shape[0], epochs, lr, seed,
                                         _p(params), ctypes.byref(loss)))
        return params, loss.value

    def selector_load_batch(self, params):
        P = np.ascontiguousarray(params, dtype=np.float32)
        _check(load().kites_selector_load_batch(self._h, _p(P), P.shape[0]))

    def selector_save_batch(self):
        P = np.empty(SELECTOR_PARAMS, dtype=np.float32)
        _check(load().kites_selector_save_batch(self._h, _p(P), SELECTOR_PARAMS))
        return P


class Graph:
    """A device-resident graph (kites::graph_csr_device)."""

    def __init__(self, engine: Engine, R, C, E=None, V=None, frontier=None,
                 frontier_nbits=0, vpg=1, directed=True, dir_R=None, dir_C=None,
                 on_device=False, n_vertices=None, n_edges=None,
                 vertex_value_size=4, offsets64=False):
        self.engine = engine
        v = CscView()
        if on_device:
            v.n_vertices = int(n_vertices)
            v.n_edges = int(n_edges)
            r_is64 = R.dtype.itemsize == 8 if hasattr(R, "dtype") else True
        else:
            R = np.ascontiguousarray(R)
            C = np.ascontiguousarray(C, dtype=np.uint32)
            v.n_vertices = R.shape[0] - 1
            v.n_edges = C.shape[0]
            r_is64 = R.dtype.itemsize == 8
            if E is not None:
                E = np.ascontiguousarray(E)
            if V is not None:
                V = np.ascontiguousarray(V)
            if frontier is not None:
                frontier = np.ascontiguousarray(frontier, dtype=np.uint32)
            if dir_R is not None:
                dir_R = np.ascontiguousarray(dir_R)
                dir_C = np.ascontiguousarray(dir_C, dtype=np.uint32)
        if r_is64:
            v.row_offsets = _p(R)
        else:
            v.row_offsets32 = _p(R)
        v.col_indices = _p(C)
        v.edge_values = _p(E)
        v.edge_value_size = 0 if E is None else 4
        v.vertex_value_size = vertex_value_size
        v.vertex_values = _p(V)
        v.vertex_per_group = vpg
        v.directed = 1 if directed else 0
        v.frontier_bits = _p(frontier)
        v.frontier_nbits = int(frontier_nbits)
        if dir_R is not None:
            v.n_out_rows = dir_R.shape[0] - 1
            if dir_R.dtype.itemsize == 8:
                v.out_row_offsets = _p(dir_R)
            else:
                v.out_row_offsets32 = _p(dir_R)
            v.out_col_indices = _p(dir_C)
            v.n_out_edges = dir_C.shape[0]
        v.on_device = 1 if on_device else 0
        v.offsets64 = 1 if offsets64 else 0
        self._keep = (R, C, E, V, frontier, dir_R, dir_C)
        self._h = c_void_p()
        _check(load().kites_graph_upload(engine._h, ctypes.byref(v), ctypes.byref(self._h)))
        engine._graphs.add(self)
        self._keep = None
        self.n_vertices = int(v.n_vertices)
        self.n_edges = int(v.n_edges)
        dv = self.device_view()
        self.n_padded = int(dv.n_vertices)

    @classmethod
    def from_edges(cls, engine: Engine, n_vertices, src, dst, w=None, directed=True):
        """CSC built on the device from an edge list (kites_graph_from_edges);
        src/dst/w are numpy arrays or device pointers with n_edges given by
        len(src)."""
        self = cls.__new__(cls)
        self.engine = engine
        if hasattr(src, "ctypes"):
            src = np.ascontiguousarray(src, dtype=np.uint32)
            dst = np.ascontiguousarray(dst, dtype=np.uint32)
            if w is not None:
                w = np.ascontiguousarray(w, dtype=np.uint32)
        m = len(src)
        self._keep = None
        self._h = c_void_p()
        _check(load().kites_graph_from_edges(engine._h, int(n_vertices), m, _p(src), _p(dst),
                                             _p(w), 1 if directed else 0,
                                             ctypes.byref(self._h)))
        engine._graphs.add(self)
        self.n_vertices = int(n_vertices)
        self.n_edges = m
        self.n_padded = int(self.device_view().n_vertices)
        return self

    def close(self):
        if self._h:
            if self.engine._h:
                load().kites_graph_destroy(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_view(self) -> DeviceView:
        dv = DeviceView()
        _check(load().kites_graph_device_view(self._h, ctypes.byref(dv)))
        return dv

    def get_values(self, n=None, dtype=np.uint32):
        n = self.n_padded if n is None else n
        out = np.empty(n, dtype=dtype)
        _check(load().kites_graph_get_values(self._h, _p(out), n))
        return out

    def set_values(self, values):
        values = np.ascontiguousarray(values)
        _check(load().kites_graph_set_values(self._h, _p(values), values.shape[0]))

    def set_frontier(self, bits, nbits):
        bits = np.ascontiguousarray(bits, dtype=np.uint32)
        _check(load().kites_graph_set_frontier(self._h, _p(bits), nbits))

    # ---- runs ----
    def process(self, op, opts=None):
        st = RunStats()
        o = opts or default_opts()
        _check(load().kites_process(self.engine._h, self._h, op, ctypes.byref(o),
                                    ctypes.byref(st)))
        return st

    def sssp(self, source, op=OP_SSSP, out=None, opts=None):
        """out=None: new host array; out=False: leave the distances on the
        device (graph values); otherwise a host/device buffer of n values."""
        st = RunStats()
        o = opts or default_opts()
        if out is None:
            out = np.empty(self.n_vertices, dtype=np.uint32)
        ptr = None if out is False else _p(out)
        _check(load().kites_sssp(self.engine._h, self._h, op, source, ptr,
                                 ctypes.byref(o), ctypes.byref(st)))
        return (None if out is False else out), st

    def sssp_batch(self, sources, op=OP_SSSP, out=None, opts=None):
        st = RunStats()
        o = opts or default_opts()
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        k = src.shape[0]
        if out is None:
            out = np.empty((self.n_vertices, k), dtype=np.uint32)
        _check(load().kites_sssp_batch(self.engine._h, self._h, op, _p(src), k, _p(out),
                                       ctypes.byref(o), ctypes.byref(st)))
        return out, st

    def sssp_multi_seed(self, seeds, op=OP_SSSP, out=None, opts=None):
        st = RunStats()
        o = opts or default_opts()
        sd = np.ascontiguousarray(seeds, dtype=np.uint32)
        if out is None:
            out = np.empty(self.n_vertices, dtype=np.uint32)
        ptr = None if out is False else _p(out)
        _check(load().kites_sssp_multi_seed(self.engine._h, self._h, op, _p(sd), sd.shape[0],
                                            ptr, ctypes.byref(o), ctypes.byref(st)))
        return (None if out is False else out), st

    def selector_record(self, op=OP_SSSP, source=0, capacity=512):
        """Per iteration: 12 features and the time (ms) of each selector class."""
        X = np.zeros((capacity, SELECTOR_FEATURES), dtype=np.float32)
        T = np.zeros((capacity, SELECTOR_CLASSES), dtype=np.float32)
        n = c_uint32()
        _check(load().kites_selector_record(self.engine._h, self._h, op, source, _p(X), _p(T),
                                            capacity, ctypes.byref(n)))
        return X[: n.value], T[: n.value]

    def selector_record_batch(self, sources, op=OP_SSSP, capacity=512):
        """Per iteration of a batched run: 12 features and the time (ms) of
        each batched class (PLAIN, PUSH, PULL_ALL, PULL_CHANGED)."""
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        X = np.zeros((capacity, SELECTOR_FEATURES), dtype=np.float32)
        T = np.zeros((capacity, SELECTOR_CLASSES), dtype=np.float32)
        n = c_uint32()
        _check(load().kites_selector_record_batch(self.engine._h, self._h, op, _p(src),
                                                  src.shape[0], _p(X), _p(T), capacity,
                                                  ctypes.byref(n)))
        return X[: n.value], T[: n.value]

    def set_batch_gather(self, mode):
        _check(load().kites_graph_set_batch_gather(self._h, int(mode)))

    def set_tpv(self, strategy):
        _check(load().kites_graph_set_tpv(self._h, strategy))

    def set_coarse(self, strategy):
        """The selector's coarse class: STRATEGY_PULL_ALL or STRATEGY_MIP."""
        _check(load().kites_graph_set_coarse(self._h, strategy))

    def build_mipmap(self, block_vertices):
        """Block map of the mipmapped frontier (STRATEGY_MIP), built on the device."""
        _check(load().kites_graph_build_mipmap(self._h, int(block_vertices)))

    def mipmap(self):
        """(dim, words): the block map as dim * dim / 32 uint32 words."""
        dim = c_uint64()
        _check(load().kites_graph_get_mipmap(self._h, ctypes.byref(dim), None, 0))
        words = np.zeros(dim.value * dim.value // 32, dtype=np.uint32)
        _check(load().kites_graph_get_mipmap(self._h, ctypes.byref(dim), _p(words),
                                             words.shape[0]))
        return dim.value, words

    def autotune(self, sources, batch=64, op=OP_SSSP):
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        r = TuneResult()
        _check(load().kites_autotune(self.engine._h, self._h, op, _p(src), src.shape[0], batch,
                                     ctypes.byref(r)))
        return r

    def cc(self, out=None, opts=None):
        st = RunStats()
        o = opts or default_opts()
        if out is None:
            out = np.empty(self.n_vertices, dtype=np.uint32)
        _check(load().kites_cc(self.engine._h, self._h, _p(out), ctypes.byref(o),
                               ctypes.byref(st)))
        return out, st

    def pagerank(self, n_real=None, iterations=20, damping=0.85, out=None, opts=None):
        st = RunStats()
        o = opts or default_opts()
        o.pagerank_iterations = iterations
        o.damping = damping
        n_real = self.n_vertices if n_real is None else n_real
        if out is None:
            out = np.empty(n_real, dtype=np.float32)
        _check(load().kites_pagerank(self.engine._h, self._h, n_real, _p(out),
                                     ctypes.byref(o), ctypes.byref(st)))
        return out, st


# ---------------------------------------------------------------------------
# Synthetic graphs (host)
# ---------------------------------------------------------------------------

def gen_rmat(scale, n_edges, a=0.57, b=0.19, c=0.19, seed=1, w_lo=1, w_hi=255,
             n_vertices=0):
    src = np.empty(n_edges, dtype=np.uint32)
    dst = np.empty(n_edges, dtype=np.uint32)
    w = np.empty(n_edges, dtype=np.uint32)
    _check(load().kites_gen_rmat(scale, n_vertices, n_edges, a, b, c, seed, w_lo, w_hi,
                                 _p(src), _p(dst), _p(w)))
    return src, dst, w


def gen_rmat_union(n_graphs, seed=1, v_min=1000, v_max=100000, ef_min=4, ef_max=32, w_lo=1,
                   w_hi=255):
    """Disjoint union of R-MAT graphs; returns (src, dst, w, vertex_offsets,
    edge_offsets) with global vertex ids."""
    vo = np.zeros(n_graphs + 1, dtype=np.uint64)
    eo = np.zeros(n_graphs + 1, dtype=np.uint64)
    lib = load()
    _check(lib.kites_gen_rmat_union(n_graphs, seed, v_min, v_max, ef_min, ef_max, w_lo, w_hi,
                                    _p(vo), _p(eo), None, None, None))
    m = int(eo[-1])
    src = np.empty(m, dtype=np.uint32)
    dst = np.empty(m, dtype=np.uint32)
    w = np.empty(m, dtype=np.uint32)
    _check(lib.kites_gen_rmat_union(n_graphs, seed, v_min, v_max, ef_min, ef_max, w_lo, w_hi,
                                    _p(vo), _p(eo), _p(src), _p(dst), _p(w)))
    return src, dst, w, vo, eo


def gen_er(n_vertices, n_edges, seed=1, w_lo=1, w_hi=255):
    src = np.empty(n_edges, dtype=np.uint32)
    dst = np.empty(n_edges, dtype=np.uint32)
    w = np.empty(n_edges, dtype=np.uint32)
    _check(load().kites_gen_er(n_vertices, n_edges, seed, w_lo, w_hi, _p(src), _p(dst),
                               _p(w)))
    return src, dst, w


def gen_grid(side, seed=1, w_lo=1, w_hi=1000):
    m = 4 * side * (side - 1)
    src = np.empty(m, dtype=np.uint32)
    dst = np.empty(m, dtype=np.uint32)
    w = np.empty(m, dtype=np.uint32)
    _check(load().kites_gen_grid(side, seed, w_lo, w_hi, _p(src), _p(dst), _p(w)))
    return src, dst, w


def csc_from_edges(n_vertices, src, dst, w=None):
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    m = src.shape[0]
    R = np.empty(n_vertices + 1, dtype=np.uint64)
    C = np.empty(m, dtype=np.uint32)
    E = np.empty(m, dtype=np.uint32) if w is not None else None
    if w is not None:
        w = np.ascontiguousarray(w, dtype=np.uint32)
    _check(load().kites_csc_from_edges(n_vertices, m, _p(src), _p(dst), _p(w), _p(R),
                                       _p(C), _p(E)))
    return R, C, E


# ---------------------------------------------------------------------------
# Binary CSC files (kites_csc_save / kites_csc_info / kites_csc_load)
# ---------------------------------------------------------------------------

def csc_save(path, R, C, E=None, directed=True, desc=""):
    R = np.ascontiguousarray(R, dtype=np.uint64)
    C = np.ascontiguousarray(C, dtype=np.uint32)
    if E is not None:
        E = np.ascontiguousarray(E, dtype=np.uint32)
    _check(load().kites_csc_save(os.fsencode(path), R.shape[0] - 1, C.shape[0], _p(R), _p(C),
                                 _p(E), 1 if directed else 0, desc.encode()))


def csc_info(path):
    """(n_vertices, n_edges, has_values, directed, desc) of a CSC file."""
    n, m, hv, dr = c_uint64(), c_uint64(), c_int(), c_int()
    buf = ctypes.create_string_buffer(96)
    _check(load().kites_csc_info(os.fsencode(path), ctypes.byref(n), ctypes.byref(m),
                                 ctypes.byref(hv), ctypes.byref(dr), buf, 96))
    return n.value, m.value, bool(hv.value), bool(dr.value), buf.value.decode()


def csc_load(path):
    """(R uint64, C, E or None) of a CSC file."""
    n, m, hv, _, _ = csc_info(path)
    R = np.empty(n + 1, dtype=np.uint64)
    C = np.empty(m, dtype=np.uint32)
    E = np.empty(m, dtype=np.uint32) if hv else None
    _check(load().kites_csc_load(os.fsencode(path), _p(R), _p(C), _p(E)))
    return R, C, E
