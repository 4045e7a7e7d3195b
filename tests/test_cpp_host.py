"""The host-side construction of the kites:: C++ front-end, on the CPU.

tests/cpp/host_graphs.cpp builds kites::graph_csr (vertex groups 1 to 64,
directed and undirected) and kites::graph_csr_mipmapped (block sizes 1, 3,
32, 100) from the config-1 edge list and the reference example's Wiki-Vote
file with g++, linked against host-memory stand-ins for the
four CUDA runtime calls the host buffers make (tests/cpp/host_runtime_stub.cpp),
and every array must hash to the golden value the reference's own classes
produced (tests/golden/make_golden.py)."""
import hashlib
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.digest()


@pytest.fixture(scope="module")
def tool(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("hg") / "host_graphs")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    "-I", "/usr/local/cuda/include", "-o", exe,
                    os.path.join(CPP, "host_graphs.cpp"), os.path.join(CPP, "host_runtime_stub.cpp")],
                   check=True, capture_output=True)
    return exe


@pytest.fixture(scope="module")
def cfg1_file(cfg1_edges, tmp_path_factory):
    s, d, w = cfg1_edges
    path = tmp_path_factory.mktemp("cfg1") / "edges.txt"
    with open(path, "w") as f:
        for a, b, c in zip(s.tolist(), d.tolist(), w.tolist()):
            f.write(f"{a}\t{b}\t{c}\n")
    return str(path)


def dump(tool, mode, edges, param, out, source=0):
    subprocess.run([tool, mode, edges, str(param), str(source), str(out)], check=True,
                   capture_output=True)
    with open(out, "rb") as f:
        counts = [int(x) for x in np.frombuffer(f.read(56), np.uint64)]
        return [np.frombuffer(f.read(4 * k), np.uint32) for k in counts[:6 if mode == "mip" else 7]], counts


@pytest.mark.parametrize("vpg", [1, 2, 4, 8])
def test_graph_csr_matches_reference(tool, cfg1_file, golden, tmp_path, vpg):
    (V, R, C, E, bits, dR, dC), _ = dump(tool, "csr", cfg1_file, vpg, tmp_path / "d.bin")
    assert sha(R, C, E, V, bits, dR, dC) == bytes(golden[f"cfg1_struct_vpg{vpg}"])


@pytest.mark.parametrize("cr", [1, 3, 32, 100])
def test_graph_csr_mipmapped_matches_reference(tool, cfg1_file, golden, tmp_path, cr):
    (V, R, C, E, bits, mip), counts = dump(tool, "mip", cfg1_file, cr, tmp_path / "d.bin")
    assert counts[6] == golden["meta"]["cfg1_mipmap_dim"][str(cr)]
    assert sha(V, R, C, E, bits, mip) == bytes(golden[f"cfg1_mipmap_cr{cr}"])


@pytest.mark.parametrize("vpg", [1, 2, 4, 8, 32, 64])
def test_graph_csr_matches_reference_wiki(tool, golden, has_reference, tmp_path, vpg):
    """The reference example's graph (Wiki-Vote, source 30, INF 2^30 - 1,
    weights (s + 1)(d + 2) % 127) at every vertex-group size the reference
    allows."""
    if not has_reference:
        pytest.skip("reference example file not present")
    from conftest import WIKI
    (V, R, C, E, bits, dR, dC), _ = dump(tool, "csr", WIKI, vpg, tmp_path / "d.bin", source=30)
    assert sha(R, C, E, V, bits, dR, dC) == bytes(golden[f"wiki_struct_vpg{vpg}"])


def test_graph_csr_undirected_matches_reference_wiki(tool, golden, has_reference, tmp_path):
    if not has_reference:
        pytest.skip("reference example file not present")
    from conftest import WIKI
    (V, R, C, E, bits, dR, dC), _ = dump(tool, "undir", WIKI, 1, tmp_path / "d.bin", source=30)
    assert dR.size == 0 and dC.size == 0 and not bits.any()
    assert sha(R, C, E, V, bits, dR, dC) == bytes(golden["wiki_undir_struct"])


@pytest.mark.parametrize("cr", [1, 3, 32, 100])
def test_graph_csr_mipmapped_matches_reference_wiki(tool, golden, has_reference, tmp_path, cr):
    if not has_reference:
        pytest.skip("reference example file not present")
    from conftest import WIKI
    (V, R, C, E, bits, mip), counts = dump(tool, "mip", WIKI, cr, tmp_path / "d.bin", source=30)
    assert counts[6] == golden["meta"]["wiki"]["mipmap_dim"][str(cr)]
    assert sha(V, R, C, E, bits, mip) == bytes(golden[f"wiki_mipmap_cr{cr}"])



def test_prepared_format_matches_reference(tool, cfg1_file, golden, tmp_path):
    """kites::io::save_to_file writes the reference's prepared text format
    byte for byte (kites/io/graph_output.cuh:23-31)."""
    out = tmp_path / "prepared.txt"
    subprocess.run([tool, "save", cfg1_file, "1", "0", str(out)], check=True, capture_output=True)
    assert hashlib.sha256(out.read_bytes()).digest() == bytes(golden["cfg1_prepared_sha"])


def test_prepared_format_round_trip(tool, cfg1_file, golden, tmp_path):
    """graph_csr(prepared file) reads back the graph that was saved
    (kites/graph/graph_csr.h:112-166)."""
    prepared = tmp_path / "prepared.txt"
    subprocess.run([tool, "save", cfg1_file, "1", "0", str(prepared)], check=True,
                   capture_output=True)
    (V, R, C, E, bits, dR, dC), _ = dump(tool, "load", str(prepared), 1, tmp_path / "d.bin")
    assert sha(R, C, E, V, bits, dR, dC) == bytes(golden["cfg1_struct_vpg1"])


def test_sanity_check_agrees_with_reference_wiki(tool, golden, has_reference, tmp_path):
    """kites::sanity_check (the reference's CPU verifier, kites/graph/sanity_check.cuh:13-59)
    passes on the reference's fixed point of the example graph after the same number of
    Gauss-Seidel sweeps, and reports the first mismatch of a perturbed result."""
    if not has_reference:
        pytest.skip("reference example file not present")
    from conftest import WIKI
    want = golden["wiki_sssp"].astype(np.uint32)
    vf = tmp_path / "v.bin"
    vf.write_bytes(want.tobytes())
    r = subprocess.run([tool, "check", WIKI, "1", "30", str(vf)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "SANITY CHECK: PASSED" in r.stdout
    sweeps = golden["meta"]["wiki"]["sweeps"]
    assert f"performed {sweeps} iterations" in r.stdout
    bad = want.copy()
    i = int(np.flatnonzero(bad < 1000)[3])
    bad[i] += 1
    vf.write_bytes(bad.tobytes())
    r = subprocess.run([tool, "check", WIKI, "1", "30", str(vf)], capture_output=True, text=True)
    assert r.returncode == 5 and f"MISMATCH at index {i}" in r.stdout


def test_sanity_check_agrees_with_oracle_cfg1(tool, cfg1_file, tmp_path):
    vals = np.loadtxt(cfg1_file, dtype=np.int64).astype(np.uint32)
    hg = O.build_host_graph(vals[:, 0], vals[:, 1], vals[:, 2], init="source", source=0,
                            inf=1073741823)
    want, _ = O.sanity_check(hg, op=O.OP_SSSP_WRAP)
    vf = tmp_path / "v.bin"
    vf.write_bytes(np.asarray(want, np.uint32).tobytes())
    r = subprocess.run([tool, "check", cfg1_file, "1", "0", str(vf)], capture_output=True,
                       text=True)
    assert r.returncode == 0 and "SANITY CHECK: PASSED" in r.stdout
