"""Binary CSC files read and written with numpy alone -- TEST INFRASTRUCTURE.

A restatement of the file layout the library writes (kites_csc_save in
include/kites_b200.h): a 128-byte header ("KITESCSC", uint32 version 1,
uint32 flags with 1 = edge values and 2 = directed, uint64 n_vertices,
uint64 n_edges, uint64 0, 88 bytes of NUL-padded description), then R as
n_vertices + 1 uint64, C and E as n_edges uint32 each.  The benchmark's
reference arm reads its input graph with this module, so it never loads the
product library; the tests check that both sides read each other's files.
"""
from __future__ import annotations

import os

import numpy as np

MAGIC = b"KITESCSC"
HEADER = np.dtype([("magic", "S8"), ("version", "<u4"), ("flags", "<u4"),
                   ("n_vertices", "<u8"), ("n_edges", "<u8"), ("reserved", "<u8"),
                   ("desc", "S88")])
assert HEADER.itemsize == 128


def read_header(path):
    """(n_vertices, n_edges, has_values, directed, desc); raises ValueError on
    a file that is not a complete version-1 CSC file."""
    with open(path, "rb") as f:
        raw = f.read(HEADER.itemsize)
    if len(raw) != HEADER.itemsize:
        raise ValueError(f"{path}: shorter than a CSC header")
    h = np.frombuffer(raw, dtype=HEADER)[0]
    if h["magic"] != MAGIC or int(h["version"]) != 1:
        raise ValueError(f"{path} is not a version-1 CSC file")
    n, m, flags = int(h["n_vertices"]), int(h["n_edges"]), int(h["flags"])
    want = HEADER.itemsize + 8 * (n + 1) + 4 * m * (2 if flags & 1 else 1)
    if os.path.getsize(path) != want:
        raise ValueError(f"{path} is truncated or has trailing bytes")
    return n, m, bool(flags & 1), bool(flags & 2), h["desc"].decode()


def read(path):
    """(R uint64, C uint32, E uint32 or None, directed, desc)."""
    n, m, has_e, directed, desc = read_header(path)
    with open(path, "rb") as f:
        f.seek(HEADER.itemsize)
        R = np.fromfile(f, dtype="<u8", count=n + 1)
        C = np.fromfile(f, dtype="<u4", count=m)
        E = np.fromfile(f, dtype="<u4", count=m) if has_e else None
    if R[0] != 0 or int(R[-1]) != m:
        raise ValueError(f"{path}: R does not span 0 .. n_edges")
    return R, C, E, directed, desc


def write(path, R, C, E=None, directed=True, desc=""):
    """Writes under a temporary name, then renames into place."""
    R = np.ascontiguousarray(R, dtype="<u8")
    C = np.ascontiguousarray(C, dtype="<u4")
    h = np.zeros(1, dtype=HEADER)
    h["magic"] = MAGIC
    h["version"] = 1
    h["flags"] = (1 if E is not None else 0) | (2 if directed else 0)
    h["n_vertices"] = R.shape[0] - 1
    h["n_edges"] = C.shape[0]
    h["desc"] = desc.encode()[:87]
    tmp = f"{path}.tmp{os.getpid()}"
    with open(tmp, "wb") as f:
        h.tofile(f)
        R.tofile(f)
        C.tofile(f)
        if E is not None:
            np.ascontiguousarray(E, dtype="<u4").tofile(f)
    os.replace(tmp, path)
