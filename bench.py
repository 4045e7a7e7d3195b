"""SSSP throughput of the B200 engine on a seeded R-MAT graph.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): directed R-MAT scale 24 -- 16,777,216 vertices,
268,435,456 edges after removing self-loops and duplicate pairs
(a,b,c,d = 0.57,0.19,0.19,0.05, seed 1), uint32 weights uniform in [1,255].
One step = single-source SSSP from each of 16 seeded sources.  The metric is
Graph500-style GTEPS: the sum over sources of edges whose source endpoint is
reached, divided by the time.  The CSC (2.2 GB) is larger than L2, so every
step streams it from HBM.

Multi-GPU: replicas only -- each rank runs its own 16 sources on its own
copy of the graph (weak scaling); torch.distributed carries only the
barrier and the max-over-ranks of the timings.

--impl reference times farkhor/KiTES's own CPU vertex-centric loop
(kites::sanity_check, compiled from the reference headers into
oracle/_ref/libref_harness.so) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SSSP GTEPS (Graph500-style, sum over sources of reached edges / time)"
UNIT = "GTEPS"
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_harness.so")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--sources", type=int, default=16)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--ref-sample-scale", type=int, default=20)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def make_graph(scale, edge_factor, seed):
    from kites_b200 import capi
    n = 1 << scale
    m = edge_factor * n
    s, d, w = capi.gen_rmat(scale, m, 0.57, 0.19, 0.19, seed, 1, 255)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    outdeg = np.bincount(s, minlength=n).astype(np.uint64)
    del s, d, w
    return n, m, R, C, E, outdeg


def pick_sources(outdeg, count, seed, offset=0):
    """Seeded sources among vertices with out-edges (SplitMix64 draws)."""
    cand = np.flatnonzero(outdeg > 0)
    out = []
    k = offset * 1000
    mask = (1 << 64) - 1
    while len(out) < count:
        z = (seed * 0x9E3779B97F4A7C15 + (k + 1) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z ^= z >> 31
        v = int(cand[z % cand.shape[0]])
        if v not in out:
            out.append(v)
        k += 1
    return np.array(out, dtype=np.uint32)


def reached_edges(dist, outdeg):
    return int(outdeg[: dist.shape[0]][dist != 0xFFFFFFFF].sum())


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(backend):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as tdist
        tdist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x, world, device):
    if world == 1:
        return x
    import torch
    import torch.distributed as tdist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world, device):
    if world == 1:
        return x
    import torch
    import torch.distributed as tdist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.SUM)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as tdist
        tdist.barrier()


# ---------------------------------------------------------------------------
# reference CPU arm
# ---------------------------------------------------------------------------

def ref_sample(scale, seed, sources=1):
    """Bounded sample for the reference's single-thread loop: SSSP from one
    seeded source on an R-MAT of `scale` with the same generator and
    parameters as the benchmark graph."""
    n, m, R, C, E, outdeg = make_graph(scale, 16, seed)
    if R[-1] > 0xFFFFFFFF:
        raise RuntimeError("reference loop takes 32-bit offsets")
    srcs = pick_sources(outdeg, sources, seed)
    return n, m, R.astype(np.uint32), C, E, outdeg, srcs


def time_reference(lib, n, m, R32, C, E, outdeg, src):
    V = np.full(n, 0xFFFFFFFF, np.uint32)
    V[src] = 0
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    secs = lib.ref_sanity_check_csc(0, n, m, p(V), p(R32), p(C), p(E))
    if secs < 0:
        raise RuntimeError("reference loop failed")
    return secs, reached_edges(V, outdeg)


def load_ref_lib():
    if not os.path.exists(REF_LIB):
        return None
    lib = ctypes.CDLL(REF_LIB)
    lib.ref_sanity_check_csc.restype = ctypes.c_double
    lib.ref_sanity_check_csc.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64] + \
        [ctypes.c_void_p] * 4
    return lib


def run_reference(args):
    world, rank, _ = dist_setup("gloo")
    config = workload_config(args)
    if rank != 0:
        return 0
    lib = load_ref_lib()
    if lib is None:
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libref_harness.so not built "
                                         "(needs the reference tree at build time)"}))
        return 0
    n, m, R32, C, E, outdeg, srcs = ref_sample(args.ref_sample_scale, args.seed,
                                               args.warmup + args.steps)
    times, edges = [], []
    for i in range(args.warmup + args.steps):
        secs, me = time_reference(lib, n, m, R32, C, E, outdeg, int(srcs[i]))
        if i >= args.warmup:
            times.append(secs)
            edges.append(me)
    total_t = sum(times)
    value = sum(edges) / total_t / 1e9
    sample = (f"single-source SSSP per step on R-MAT scale {args.ref_sample_scale} "
              f"({n} vertices, {m} edges, same generator/parameters), one seeded "
              f"source per step, reference kites::sanity_check loop, 1 thread")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_t / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": config,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))
    return 0


def workload_config(args):
    n = 1 << args.scale
    return {"workload": f"sssp_rmat_scale{args.scale}",
            "graph": f"directed R-MAT scale {args.scale}: {n} vertices, "
                     f"{args.edge_factor * n} edges, a,b,c=0.57,0.19,0.19, seed {args.seed}, "
                     f"uint32 weights U[1,255], no self-loops/duplicates",
            "sources_per_step": args.sources, "strategy": "plain",
            "l2": "inputs larger than L2 (CSC 2.2 GB vs 126 MB L2)",
            "parallelism": f"replicas{args.gpus}"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def run_ours(args):
    import torch

    from kites_b200 import capi

    world, rank, local = dist_setup("nccl")
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    n, m, R, C, E, outdeg = make_graph(args.scale, args.edge_factor, args.seed)
    eng = capi.Engine(local)
    g = capi.Graph(eng, R, C, E)
    del C, E
    stream = torch.cuda.ExternalStream(g.device_view().stream, device=device)
    srcs = pick_sources(outdeg, args.sources, args.seed, offset=rank)
    opts = capi.default_opts(device_loop=1)

    # Warm-up (also fixes the reached-edge count per source).
    reached = np.zeros(len(srcs), np.int64)
    host_dist = np.empty(n, np.uint32)
    for w in range(args.warmup):
        for i, s in enumerate(srcs):
            dist, st = g.sssp(int(s), out=host_dist if w == 0 else False, opts=opts)
            if w == 0:
                reached[i] = reached_edges(dist, outdeg)
    units_per_step = int(reached.sum())

    # Timed region: K steps, inputs resident, events on the engine stream.
    launches = 0
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        iters = 0
        for _ in range(args.steps):
            for s in srcs:
                _, st = g.sssp(int(s), out=False, opts=opts)
                launches += st.kernel_launches
                iters += st.iterations
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, world, device)
    total_units = sum_over_ranks(units_per_step * args.steps, world, device)
    value = total_units / (ms_max * 1e-3) / 1e9

    # Roofline of the dominant kernel (k_pull_chunked): host loop with CUDA
    # events around every pull launch, one pass over the step's sources.
    kopts = capi.default_opts(device_loop=0, time_kernels=1)
    k_ms, k_bytes, k_launch, all_bytes, dev_ms = 0.0, 0, 0, 0, 0.0
    for s in srcs:
        _, st = g.sssp(int(s), out=False, opts=kopts)
        k_ms += st.pull_kernel_ms
        k_bytes += st.pull_kernel_bytes
        k_launch += st.pull_kernel_launches
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) \
        if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = k_bytes / (k_ms * 1e-3) / 1e9 if k_ms > 0 else None
    traffic = None
    prof = os.path.join(ROOT, "profiles", "pull_traffic.json")
    if os.path.exists(prof):
        try:
            t = json.load(open(prof))
            if t.get("workload") == f"rmat{args.scale}":
                traffic = t.get("bytes_per_launch")
        except (OSError, ValueError):
            traffic = None

    # End-to-end through the C ABI: results copied to pinned host memory
    # every run (the step's inputs are the 16 source ids).
    e2e = None
    if not args.no_e2e:
        pinned = torch.empty(n, dtype=torch.int32, pin_memory=True)
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            for s in srcs:
                g.sssp(int(s), out=pinned, opts=opts)
        e1.record(stream)
        torch.cuda.synchronize()
        e_ms = max_over_ranks(e0.elapsed_time(e1), world, device)
        e2e = {"value": total_units / (e_ms * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": 4 * len(srcs),
               "d2h_bytes_per_step": 4 * n * len(srcs)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        lib = load_ref_lib()
        if lib is not None:
            n2, m2, R32, C2, E2, od2, s2 = ref_sample(args.ref_sample_scale, args.seed, 1)
            secs, me = time_reference(lib, n2, m2, R32, C2, E2, od2, int(s2[0]))
            cpu = {"value": me / secs / 1e9, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"single-source SSSP on R-MAT scale {args.ref_sample_scale} "
                             f"({n2} vertices, {m2} edges, same generator/parameters), "
                             f"reference kites::sanity_check loop, 1 thread, {secs:.2f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": workload_config(args),
            "clocks": {k: v for k, v in clk.summary().items()},
            "e2e": e2e,
            "gpu_launches": int(launches),
            "iterations_per_source": iters / (args.steps * len(srcs)),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic, "kernel": "k_pull_chunked",
                         "launches": k_launch, "peak_source": "MEASURED_PEAKS.json hbm_gbs"
                         if peaks else "fallback 6.65 TB/s"},
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    g.close()
    eng.close()
    if world > 1:
        import torch.distributed as tdist
        tdist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
