"""Regenerates tests/golden/golden.npz from farkhor/KiTES's OWN host code.

    python tests/golden/make_golden.py [--ref <reference tree>]

Needs the reference tree (only in the development container) and the
harness built from it (`make -C oracle ref`).  Every vector here comes out
of the reference's graph_csr construction and its sanity_check loop
(kites/graph/graph_csr.h, kites/graph/sanity_check.cuh) run by
oracle/_ref/ref_harness; the synthetic graphs come from this repository's
seeded generators, whose edge lists are pinned by hash.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from kites_b200 import capi  # noqa: E402  (generators only)
from oracle import oracle as O  # noqa: E402
from oracle.reference_dir import REFERENCE_DIR  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
OUT = os.path.join(ROOT, "tests", "golden", "golden.npz")

MIPMAP_CRS = (1, 3, 32, 100)
CFG1 = dict(scale=13, n_vertices=7115, n_edges=103689, a=0.57, b=0.19, c=0.19,
            seed=1, w_lo=1, w_hi=63)


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def load_build_dump(path):
    with open(path, "rb") as f:
        hdr = np.frombuffer(f.read(64), np.uint64)
        n, m, nbits, nwords, ndr, ndc, directed, vpg = (int(x) for x in hdr)

        def rd(k):
            return np.frombuffer(f.read(4 * k), np.uint32).copy()
        d = dict(n=n, m=m, nbits=nbits, directed=directed, vpg=vpg)
        d["V"], d["R"], d["C"], d["E"] = rd(n), rd(n + 1), rd(m), rd(m)
        d["bitmap"], d["dir_R"], d["dir_C"], d["Vfix"] = rd(nwords), rd(ndr), rd(ndc), rd(n)
    return d


def struct_hash(d):
    return sha(d["R"], d["C"], d["E"], d["V"], d["bitmap"], d["dir_R"], d["dir_C"])


def run_build(edge_file, vpg, source, init="sssp", directed=True, inf=None):
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "dump.bin")
        cmd = [HARNESS, "build", edge_file, str(vpg), "sd", str(source), init,
               "dir" if directed else "undir", out]
        if inf is not None:
            cmd.append(str(inf))
        log = subprocess.run(cmd, check=True, capture_output=True, text=True).stdout
        d = load_build_dump(out)
    sweeps = [int(line.split("performed")[1].split()[0]) for line in log.splitlines()
              if "performed" in line]
    d["sweeps"] = sweeps[0] if sweeps else -1
    return d


def run_mipmap(edge_file, cr, source):
    """The reference's graph_csr_mipmapped (SSSP values from `source`):
    (mipmapDim, sha256 of V, R, C, E, block frontier words, mipmap words)."""
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "dump.bin")
        subprocess.run([HARNESS, "mipmap", edge_file, str(cr), "sd", str(source), out],
                       check=True, capture_output=True)
        with open(out, "rb") as f:
            n, m, _, dim, nb, nm = (int(x) for x in np.frombuffer(f.read(48), np.uint64))
            arrays = [np.frombuffer(f.read(4 * k), np.uint32) for k in (n, n + 1, m, m, nb, nm)]
    return dim, sha(*arrays)


def run_save(edge_file, vpg, source):
    """sha256 of the reference's prepared text file (io::save_to_file)."""
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "prepared.txt")
        subprocess.run([HARNESS, "save", edge_file, str(vpg), str(source), out], check=True,
                       capture_output=True)
        with open(out, "rb") as f:
            return hashlib.sha256(f.read()).hexdigest()


def run_csc(R, C, E, V, op):
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(inp, "wb") as f:
            f.write(np.array([V.shape[0], C.shape[0]], np.uint64).tobytes())
            f.write(V.astype(np.uint32).tobytes())
            f.write(R.astype(np.uint32).tobytes())
            f.write(C.astype(np.uint32).tobytes())
            f.write((E if E is not None else np.ones_like(C)).astype(np.uint32).tobytes())
        subprocess.run([HARNESS, "csc", inp, op, out], check=True, capture_output=True)
        with open(out, "rb") as f:
            f.read(8)
            return np.frombuffer(f.read(), np.uint32).copy()


def write_edges(path, src, dst, w=None):
    with open(path, "w") as f:
        if w is None:
            for s, d in zip(src.tolist(), dst.tolist()):
                f.write(f"{s}\t{d}\n")
        else:
            for s, d, x in zip(src.tolist(), dst.tolist(), w.tolist()):
                f.write(f"{s}\t{d}\t{x}\n")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=REFERENCE_DIR,
                    help="reference tree (default: KITES_REFERENCE_DIR)")
    args = ap.parse_args(argv)
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), f"REF={args.ref}", "all"],
                   check=True, capture_output=True)
    wiki = os.path.join(args.ref, "examples", "Sample-Graph-Wiki-Vote.txt")
    g = {}
    meta = {"cfg1": CFG1, "wiki": {"source": 30, "inf": 1073741823}}

    # 1. The reference example: Wiki-Vote, SSSP from 30, INF 2^30-1,
    #    weights (s+1)(d+2)%127, vpg 1..64 (graph_csr.h:220-230).
    for vpg in (1, 2, 4, 8, 32, 64):
        d = run_build(wiki, vpg, 30)
        g[f"wiki_struct_vpg{vpg}"] = np.frombuffer(bytes.fromhex(struct_hash(d)), np.uint8)
        if vpg == 1:
            g["wiki_sssp"] = d["Vfix"]
            meta["wiki"]["sweeps"] = d["sweeps"]
            meta["wiki"]["n"] = d["n"]
    # Mipmapped construction (graph_csr_mipmapped.hpp:40-78), block sizes
    # 1, 3, 32 and 100.
    meta["wiki"]["mipmap_dim"] = {}
    for cr in MIPMAP_CRS:
        dim, h = run_mipmap(wiki, cr, 30)
        g[f"wiki_mipmap_cr{cr}"] = np.frombuffer(bytes.fromhex(h), np.uint8)
        meta["wiki"]["mipmap_dim"][str(cr)] = dim
    # Undirected (incomplete edge list) construction: the reference copies no
    # frontier bits (graph_csr.h:100-101), so process() leaves V untouched.
    d = run_build(wiki, 1, 30, directed=False)
    g["wiki_undir_struct"] = np.frombuffer(bytes.fromhex(struct_hash(d)), np.uint8)
    g["wiki_undir_fix"] = d["Vfix"]

    # 2. Config 1: R-MAT 7,115 / 103,689, seed 1, weights [1,63].
    s, t, w = capi.gen_rmat(CFG1["scale"], CFG1["n_edges"], CFG1["a"], CFG1["b"],
                            CFG1["c"], CFG1["seed"], CFG1["w_lo"], CFG1["w_hi"],
                            n_vertices=CFG1["n_vertices"])
    g["cfg1_edges_sha"] = np.frombuffer(bytes.fromhex(sha(s, t, w)), np.uint8)
    with tempfile.TemporaryDirectory() as td:
        ef = os.path.join(td, "cfg1.txt")
        write_edges(ef, s, t, w)
        d = run_build(ef, 1, 0)
        g["cfg1_struct_vpg1"] = np.frombuffer(bytes.fromhex(struct_hash(d)), np.uint8)
        for vpg in (2, 4, 8):
            dv = run_build(ef, vpg, 0)
            g[f"cfg1_struct_vpg{vpg}"] = np.frombuffer(bytes.fromhex(struct_hash(dv)),
                                                       np.uint8)
        # The prepared text format (kites/io/graph_output.cuh:23-31).
        g["cfg1_prepared_sha"] = np.frombuffer(bytes.fromhex(run_save(ef, 1, 0)), np.uint8)
        meta["cfg1_mipmap_dim"] = {}
        for cr in MIPMAP_CRS:
            dim, h = run_mipmap(ef, cr, 0)
            g[f"cfg1_mipmap_cr{cr}"] = np.frombuffer(bytes.fromhex(h), np.uint8)
            meta["cfg1_mipmap_dim"][str(cr)] = dim
    hg = O.build_host_graph(s, t, w, init="source", source=0, inf=O.INF32)
    V0 = np.full(hg.n_vertices, O.INF32, np.uint32)
    V0[0] = 0
    g["cfg1_sssp"] = run_csc(hg.R, hg.C, hg.E, V0, "sssp_sat")
    g["cfg1_bfs"] = run_csc(hg.R, hg.C, None, V0, "bfs")
    # CC on the symmetrised config-1 graph, labels = own id.
    ss = np.concatenate([s, t])
    tt = np.concatenate([t, s])
    keys = np.unique(ss.astype(np.uint64) << np.uint64(32) | tt)
    ss = (keys >> np.uint64(32)).astype(np.uint32)
    tt = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    hs = O.build_host_graph(ss, tt, None, init="label")
    g["cfg1_cc"] = run_csc(hs.R, hs.C, None, np.arange(hs.n_vertices, dtype=np.uint32), "cc")
    # A second SSSP source for coverage.
    V1 = np.full(hg.n_vertices, O.INF32, np.uint32)
    V1[4321] = 0
    g["cfg1_sssp_src4321"] = run_csc(hg.R, hg.C, hg.E, V1, "sssp_sat")

    g["meta"] = np.frombuffer(json.dumps(meta, sort_keys=True).encode(), np.uint8)
    np.savez_compressed(OUT, **g)
    print("wrote", OUT, {k: v.shape for k, v in g.items()})


if __name__ == "__main__":
    main()
