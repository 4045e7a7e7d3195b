"""SSSP throughput of the B200 engine on a seeded R-MAT graph.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): directed R-MAT scale 24 -- 16,777,216 vertices,
268,435,456 edges after removing self-loops and duplicate pairs
(a,b,c,d = 0.57,0.19,0.19,0.05, seed 1), uint32 weights uniform in [1,255].
One step = SSSP from 64 seeded sources.  The metric is Graph500-style
GTEPS: the sum over sources of edges whose source endpoint is reached,
divided by the time.  The CSC (2.2 GB) and the 64-wide distance array
(4.3 GB) are larger than L2, so every step streams them from HBM.

The headline value runs the 64 sources as batches (V x K vertex-major
distances, one pass per in-edge for all K sources); the same sources run
one at a time through the plain kernel are timed alongside ("plain").

Multi-GPU: replicas only -- each rank runs its own sources on its own copy
of the graph (weak scaling); torch.distributed carries only the barrier and
the max-over-ranks of the timings.

--impl reference times farkhor/KiTES's own CPU vertex-centric loop
(kites::sanity_check, compiled from the reference headers into
oracle/_ref/libref_harness.so) on a bounded sample of the workload.
"""
from __future__ import annotations

import argparse
import contextlib
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
# kites_run_opts.strategy values (include/kites_b200.h).
STRATEGIES = {"plain": 0, "auto": 1, "push": 2, "pull_all": 3, "tpv1": 4, "tpv4": 5,
              "tpv8": 6, "tpv32": 7}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--sources", type=int, default=64)
    ap.add_argument("--batch", type=int, default=64, choices=[16, 32, 64, 128, 256])
    ap.add_argument("--mode", default="batch", choices=["batch", "single"],
                    help="batch: --batch sources per pass over the edges (headline); "
                         "single: one source at a time through kites_sssp")
    ap.add_argument("--strategy", default="plain", choices=sorted(STRATEGIES),
                    help="per-iteration strategy of --mode single (batch runs plain)")
    ap.add_argument("--batch-gather", default="loads", choices=["loads", "tma"],
                    help="how the batched pull fetches source rows: register loads or "
                         "TMA tile::gather4 copies")
    ap.add_argument("--host-loop", action="store_true",
                    help="iterate from the host instead of the CUDA-graph device loop "
                         "(for kernel profilers)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip kites_autotune (batch chunk size, sweep densities, TPV width) "
                         "before the warm-up")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--ref-sample-scale", type=int, default=20)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
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
    k = offset * 100000
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
        self.lines = []

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
        for ln in self.lines:
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


def reduce_over_ranks(x, world, device, op):
    if world == 1:
        return x
    import torch
    import torch.distributed as tdist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=getattr(tdist.ReduceOp, op))
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as tdist
        tdist.barrier()


# ---------------------------------------------------------------------------
# reference CPU arm
# ---------------------------------------------------------------------------

def ref_sample(scale, seed, sources=1):
    """Bounded sample for the reference's single-thread loop: SSSP from
    seeded sources on an R-MAT of `scale` with the same generator and
    parameters as the benchmark graph."""
    n, m, R, C, E, outdeg = make_graph(scale, 16, seed)
    if R[-1] > 0xFFFFFFFF:
        raise RuntimeError("reference loop takes 32-bit offsets")
    srcs = pick_sources(outdeg, sources, seed)
    return n, m, R.astype(np.uint32), C, E, outdeg, srcs


@contextlib.contextmanager
def reference_output_silenced():
    """The reference's loop (kites::sanity_check) prints its own report and
    ends by comparing its fixed point with a second buffer, which here holds
    the initial values (the fixed point and the time are what is measured),
    so its MISMATCH line means nothing; its stdout goes to /dev/null during
    the call and C stdio is flushed there before stdout is restored."""
    sys.stdout.flush()
    saved = os.dup(1)
    null = os.open(os.devnull, os.O_WRONLY)
    os.dup2(null, 1)
    os.close(null)
    try:
        yield
    finally:
        ctypes.CDLL(None).fflush(None)
        os.dup2(saved, 1)
        os.close(saved)


def time_reference(lib, n, m, R32, C, E, outdeg, src):
    V = np.full(n, 0xFFFFFFFF, np.uint32)
    V[src] = 0
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    with reference_output_silenced():
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


def ref_sample_text(scale, n, m):
    return (f"single-source SSSP on R-MAT scale {scale} ({n} vertices, {m} edges, same "
            f"generator and parameters as the benchmark graph), one seeded source per "
            f"step, farkhor/KiTES kites::sanity_check loop, 1 thread")


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
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_t / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": config,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": ref_sample_text(args.ref_sample_scale, n, m)},
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
            "sources_per_step": args.sources, "mode": args.mode,
            "batch": args.batch if args.mode == "batch" else 1,
            "strategy": args.strategy, "batch_gather": args.batch_gather,
            "l2": "inputs larger than L2 (CSC 2.2 GB, distances 4.3 GB vs 126 MB L2)",
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
    g.set_batch_gather(1 if args.batch_gather == "tma" else 0)
    stream = torch.cuda.ExternalStream(g.device_view().stream, device=device)
    srcs = pick_sources(outdeg, args.sources, args.seed, offset=rank)
    K = args.batch
    if args.mode == "batch" and args.sources % K:
        raise SystemExit("--sources must be a multiple of --batch")
    groups = [srcs[i:i + K] for i in range(0, len(srcs), K)]
    if args.mode == "batch" and args.strategy != "plain":
        raise SystemExit("--mode batch runs the plain strategy")
    tuned = None
    if not args.no_autotune:
        r = g.autotune(srcs[:8], batch=K if args.mode == "batch" else 16)
        tuned = {"batch_chunk_items": int(r.batch_chunk_items),
                 "dense_edges": int(r.dense_edges), "dense_rows": int(r.dense_rows),
                 "tpv_strategy": int(r.tpv_strategy), "trials": int(r.trials)}
    loop = 0 if args.host_loop else 1
    bopts = capi.default_opts(device_loop=loop)
    sopts = capi.default_opts(device_loop=loop, strategy=STRATEGIES[args.strategy])
    lib = capi.load()

    def batched_step():
        launches = 0
        if args.mode == "single":
            for s in srcs:
                _, st = g.sssp(int(s), out=False, opts=sopts)
                launches += st.kernel_launches
            return launches
        for grp in groups:
            st = capi.RunStats()
            capi._check(lib.kites_sssp_batch(eng._h, g._h, capi.OP_SSSP, capi._p(grp), K, None,
                                             ctypes.byref(bopts), ctypes.byref(st)))
            launches += st.kernel_launches
        return launches

    for _ in range(args.warmup):
        batched_step()

    # Timed region: K steps, inputs resident, events on the engine stream.
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launches = 0
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            launches += batched_step()
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    ms_max = reduce_over_ranks(ms, world, device, "MAX")
    # Reached edges per source (the units of a step), from single runs after
    # the timed region, so that a kernel profiler sees the step's launches
    # first.
    host = np.empty(n, np.uint32)
    reached = np.array([reached_edges(g.sssp(int(s), out=host)[0], outdeg) for s in srcs])
    units_per_step = int(reached.sum())
    total_units = reduce_over_ranks(units_per_step * args.steps, world, device, "SUM")
    value = total_units / (ms_max * 1e-3) / 1e9

    # Plain kernel, the same sources one at a time.
    plain = None
    popts = capi.default_opts(device_loop=1)
    if not args.no_plain:
        for s in srcs[:4]:
            g.sssp(int(s), out=False, opts=popts)
        barrier(world)
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for s in srcs:
            g.sssp(int(s), out=False, opts=popts)
        p1.record(stream)
        torch.cuda.synchronize()
        pms = reduce_over_ranks(p0.elapsed_time(p1), world, device, "MAX")
        plain = {"value": reduce_over_ranks(units_per_step, world, device, "SUM") /
                 (pms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": pms}

    # Rooflines of the dominant kernels, timed live with CUDA events around
    # every launch (host loop): k_pull_batch for the headline, k_pull_chunked
    # for the plain kernel's traversal phase.
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    kopts = capi.default_opts(device_loop=0, time_kernels=1)
    b_ach, b_launch = None, 0
    if args.mode == "batch":
        st = capi.RunStats()
        capi._check(lib.kites_sssp_batch(eng._h, g._h, capi.OP_SSSP, capi._p(groups[0]), K,
                                         None, ctypes.byref(kopts), ctypes.byref(st)))
        b_ach = st.pull_kernel_bytes / (st.pull_kernel_ms * 1e-3) / 1e9
        b_launch = int(st.pull_kernel_launches)
    k_ms, k_bytes, k_launch = 0.0, 0, 0
    d_ms, d_bytes, d_launch = 0.0, 0, 0
    for s in srcs[:8]:
        _, pst = g.sssp(int(s), out=False, opts=kopts)
        k_ms += pst.pull_kernel_ms
        k_bytes += pst.pull_kernel_bytes
        k_launch += pst.pull_kernel_launches
        d_ms += pst.pull_dense_ms
        d_bytes += pst.pull_dense_bytes
        d_launch += pst.pull_dense_launches
    p_ach = k_bytes / (k_ms * 1e-3) / 1e9
    # The same restricted to the iterations whose pull ran as the dense sweep.
    d_ach = d_bytes / (d_ms * 1e-3) / 1e9 if d_ms > 0 else None
    # DRAM bytes per launch of the batched pull, from the ncu summary of the
    # same workload (one capture of every launch of a step), when there is one.
    traffic = None
    prof = os.path.join(ROOT, "profiles", f"k_pull_batch_K{K}_rmat{args.scale}_traffic.md")
    if args.mode == "batch" and os.path.exists(prof):
        import re
        m = re.search(r"DRAM bytes per launch \(read \+ write, mean\): ([0-9]+)", open(prof).read())
        traffic = int(m.group(1)) if m else None
    src_note = "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6.65 TB/s"

    # End to end through the C ABI: every batch's V x K distances copied to
    # pinned host memory (the step's inputs are its source ids).
    e2e = None
    if not args.no_e2e and args.mode == "single":
        pinned = torch.empty(n, dtype=torch.int32, pin_memory=True)
        host_view = pinned.numpy().view(np.uint32)
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            for s in srcs:
                g.sssp(int(s), out=host_view, opts=sopts)
        e1.record(stream)
        torch.cuda.synchronize()
        e_ms = reduce_over_ranks(e0.elapsed_time(e1), world, device, "MAX")
        e2e = {"value": total_units / (e_ms * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": 4 * len(srcs),
               "d2h_bytes_per_step": 4 * n * len(srcs)}
    elif not args.no_e2e:
        pinned = torch.empty((n, K), dtype=torch.int32, pin_memory=True)
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            for grp in groups:
                capi._check(lib.kites_sssp_batch(eng._h, g._h, capi.OP_SSSP, capi._p(grp), K,
                                                 capi._p(pinned), ctypes.byref(bopts), None))
        e1.record(stream)
        torch.cuda.synchronize()
        e_ms = reduce_over_ranks(e0.elapsed_time(e1), world, device, "MAX")
        e2e = {"value": total_units / (e_ms * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": 4 * len(srcs),
               "d2h_bytes_per_step": 4 * n * len(srcs)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rlib = load_ref_lib()
        if rlib is not None:
            n2, m2, R32, C2, E2, od2, s2 = ref_sample(args.ref_sample_scale, args.seed, 1)
            secs, me = time_reference(rlib, n2, m2, R32, C2, E2, od2, int(s2[0]))
            cpu = {"value": me / secs / 1e9, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": ref_sample_text(args.ref_sample_scale, n2, m2) +
                   f" ({secs:.2f} s)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": dict(workload_config(args), autotuned=tuned),
            "clocks": clk.summary(),
            "e2e": e2e,
            "gpu_launches": int(launches),
            "plain": plain,
            "speedup_vs_plain": (value / plain["value"]) if plain else None,
            "roofline": ({"bound": "hbm", "achieved": b_ach, "peak": peak, "unit": "GB/s",
                          "frac": b_ach / peak, "traffic": traffic,
                          "kernel": f"k_pull_batch<SSSP,K={K}>",
                          "launches": b_launch, "peak_source": src_note}
                         if b_ach is not None else
                         {"bound": "hbm", "achieved": p_ach, "peak": peak, "unit": "GB/s",
                          "frac": p_ach / peak, "traffic": None,
                          "kernel": "k_pull_chunked + k_sweep + k_sweep_changed<SSSP> (plain pull)",
                          "launches": k_launch, "peak_source": src_note}),
            "roofline_plain": {"bound": "hbm", "achieved": p_ach, "peak": peak,
                               "unit": "GB/s", "frac": p_ach / peak,
                               "kernel": "k_pull_chunked + k_sweep + k_sweep_changed<SSSP> (plain pull phase)",
                               "launches": k_launch,
                               "peak_source": src_note},
            "roofline_plain_dense": ({"bound": "hbm", "achieved": d_ach, "peak": peak,
                                      "unit": "GB/s", "frac": d_ach / peak,
                                      "kernel": "k_sweep<SSSP, row filter> + k_sweep_changed<SSSP> (dense iterations)",
                                      "launches": d_launch, "peak_source": src_note}
                                     if d_ach is not None else None),
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
