"""Builds libkites_b200.so (the C-ABI library) in-tree with nvcc for sm_100a.

    python -m kites_b200.build [--force] [-v]

Every .cu and host/*.cpp under csrc/ goes into one shared object next to
this file; objects are cached under kites_b200/_build/ by source mtime.
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libkites_b200.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
                     "-Xcompiler", "-fPIC,-fopenmp", "-I", INCLUDE, "-I", CSRC]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-I", INCLUDE, "-I", CSRC,
             "-I", "/usr/local/cuda/include"]


def _deps(src: str) -> list[str]:
    hdrs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hdrs += glob.glob(os.path.join(CSRC, "*.inc"))
    hdrs += glob.glob(os.path.join(INCLUDE, "*.h"))
    return [src] + hdrs


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        if force or _stale(obj, _deps(src)):
            cmd = [NVCC] + NVCC_FLAGS + ["-Xptxas", "-v" if verbose else "-O3",
                                         "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
        objs.append(obj)
    for src in sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp"))):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        if force or _stale(obj, _deps(src)):
            cmd = ["g++"] + CXX_FLAGS + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
        objs.append(obj)
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-Xcompiler", "-fopenmp", "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


EXAMPLES = os.path.join(ROOT, "examples")
EXAMPLE_BIN = os.path.join(EXAMPLES, "_build")
# Example programs over the C++ drop-in API that the tests and the benchmark
# run (built next to the sources, in examples/_build/).
BUILT_EXAMPLES = ["sssp_binary_csc"]


def build_examples(force: bool = False, verbose: bool = False) -> list[str]:
    build(force=force, verbose=verbose)
    os.makedirs(EXAMPLE_BIN, exist_ok=True)
    hdrs = glob.glob(os.path.join(INCLUDE, "kites", "*", "*")) + [os.path.join(INCLUDE, "kites_b200.h")]
    out = []
    for name in BUILT_EXAMPLES:
        src = os.path.join(EXAMPLES, name + ".cu")
        exe = os.path.join(EXAMPLE_BIN, name)
        if force or _stale(exe, [src, LIB] + hdrs):
            cmd = [NVCC] + ARCH + ["-O3", "-std=c++17", "--expt-extended-lambda", "-I", INCLUDE,
                                   src, "-o", exe, "-L", HERE, "-lkites_b200",
                                   "-Xlinker", "-rpath=$ORIGIN/../../kites_b200"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
        out.append(exe)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    for exe in build_examples(force=a.force, verbose=a.verbose):
        print(exe)
    return 0


if __name__ == "__main__":
    sys.exit(main())
