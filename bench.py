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

Input: the graph is read from a binary CSC file (kites_csc_save's layout)
in $KITES_GRAPH_CACHE (default: <tmp>/kites_graph_cache) when one with the
same description exists, and generated and written there otherwise, so that
a 268M-edge graph is built once per machine.

--impl reference times farkhor/KiTES's own CPU vertex-centric loop
(kites::sanity_check, compiled from the reference headers into
oracle/_ref/libref_harness.so) on the same graph: each step is the SSSP of
one of the workload's sources (or of threads // K of them, when the K timed
steps would leave host threads idle), and the sources run side by side, one
per host thread.  That process reads or generates the graph through the oracle only
(oracle/csc_file.py, the oracle's own generator) and never loads the
library under test.
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

METRIC = "SSSP GTEPS on 1 B200: learned+batched vs plain kernel, bit-exact; % of HBM peak"
# How the value is counted (both arms).
METRIC_DETAIL = ("Graph500-style GTEPS: the sum over sources of the edges whose source endpoint "
                 "is reached, divided by the time")
UNIT = "GTEPS"
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_harness.so")
# kites_run_opts.strategy values (include/kites_b200.h).
STRATEGIES = {"plain": 0, "auto": 1, "push": 2, "pull_all": 3, "tpv1": 4, "tpv4": 5,
              "tpv8": 6, "tpv32": 7, "pull_changed": 8, "mip": 9}


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
    ap.add_argument("--strategy", default=None, choices=sorted(STRATEGIES),
                    help="per-iteration strategy: auto = the learned selector (the default of "
                         "--mode batch: learned + batched); plain = the fixed plain kernel (the "
                         "default of --mode single); batch mode takes plain, auto, push, "
                         "pull_all and pull_changed")
    ap.add_argument("--batch-gather", default="async", choices=["loads", "tma", "async"],
                    help="how the batched pull fetches source rows: register loads, "
                         "TMA tile::gather4 copies, or cp.async copies into shared memory")
    ap.add_argument("--host-loop", action="store_true",
                    help="iterate from the host instead of the CUDA-graph device loop "
                         "(for kernel profilers)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip kites_autotune (batch chunk size, sweep densities, TPV width) "
                         "before the warm-up")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--ref-threads", type=int, default=0,
                    help="host threads of the reference loop (0 = every core this process may use)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-lambda", action="store_true",
                    help="skip the kites::process user-function leg (examples/sssp_binary_csc)")
    ap.add_argument("--lambda-sources", type=int, default=4)
    ap.add_argument("--suite", action="store_true",
                    help="instead of the headline, one JSON line per other configuration: "
                         "config 1 through kites_process, BFS / CC / PageRank, 256 sources on "
                         "R-MAT scale 20, the 1,000-graph batch, an Erdos-Renyi graph")
    ap.add_argument("--batch-selector", default=None,
                    help="load the batched selector's weights from this file (1628 float32) "
                         "instead of the compiled-in default")
    ap.add_argument("--mip-block", type=int, default=4096,
                    help="--mode single --strategy mip (or a coarse class of MIP, "
                         "--coarse mip): vertices per block of the block map")
    ap.add_argument("--coarse", default="pull_all", choices=["pull_all", "mip"],
                    help="single-source AUTO: what the selector's coarse class runs")
    ap.add_argument("--margin", type=float, default=None,
                    help="AUTO: the selector's fallback margin (kites_run_opts."
                         "selector_margin) instead of the library default")
    a = ap.parse_args()
    if a.strategy is None:
        a.strategy = "auto" if a.mode == "batch" else "plain"
    return a


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def graph_desc(scale, edge_factor, seed):
    return (f"rmat scale={scale} m={edge_factor << scale} a,b,c=0.57,0.19,0.19 "
            f"seed={seed} w=1..255 directed")


def cache_path(scale, edge_factor, seed):
    import tempfile
    d = os.environ.get("KITES_GRAPH_CACHE") or os.path.join(tempfile.gettempdir(),
                                                             "kites_graph_cache")
    os.makedirs(d, exist_ok=True)
    return os.path.join(d, f"rmat{scale}_ef{edge_factor}_seed{seed}.csc")


def make_graph(scale, edge_factor, seed):
    """The benchmark graph through the library: read from the CSC cache when
    it holds this graph, else generated (kites_gen_rmat + kites_csc_from_edges)
    and written there (kites_csc_save)."""
    from kites_b200 import capi
    n = 1 << scale
    m = edge_factor * n
    path, desc = cache_path(scale, edge_factor, seed), graph_desc(scale, edge_factor, seed)
    R = None
    try:
        if capi.csc_info(path)[4] == desc:
            R, C, E = capi.csc_load(path)
    except capi.KitesError:
        R = None
    if R is None:
        s, d, w = capi.gen_rmat(scale, m, 0.57, 0.19, 0.19, seed, 1, 255)
        R, C, E = capi.csc_from_edges(n, s, d, w)
        del s, d, w
        capi.csc_save(path, R, C, E, directed=True, desc=desc)
    outdeg = np.bincount(C, minlength=n).astype(np.uint64)
    return n, m, R, C, E, outdeg


def make_graph_oracle(scale, edge_factor, seed):
    """The same graph for the reference arm, through the oracle alone: read
    with numpy (oracle/csc_file.py), or generated by the oracle's own
    restatement of the generator rule and written to the same cache."""
    from oracle import csc_file
    from oracle import oracle as O
    n = 1 << scale
    m = edge_factor * n
    path, desc = cache_path(scale, edge_factor, seed), graph_desc(scale, edge_factor, seed)
    R = None
    try:
        R, C, E, _, got = csc_file.read(path)
        if got != desc:
            R = None
    except (OSError, ValueError):
        R = None
    if R is None:
        s, d, w = O.gen_rmat(scale, m, 0.57, 0.19, 0.19, seed, 1, 255)
        R, C, E = O.csc_from_edges(n, s, d, w)
        del s, d, w
        csc_file.write(path, R, C, E, directed=True, desc=desc)
    outdeg = np.bincount(C, minlength=n).astype(np.uint64)
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


def host_threads(requested=0):
    return requested or len(os.sched_getaffinity(0))


def load_ref_lib():
    if not os.path.exists(REF_LIB):
        return None
    lib = ctypes.CDLL(REF_LIB)
    lib.ref_sssp_sources.restype = ctypes.c_double
    lib.ref_sssp_sources.argtypes = [ctypes.c_uint64, ctypes.c_uint64] + [ctypes.c_void_p] * 4 + \
        [ctypes.c_uint32, ctypes.c_uint32] + [ctypes.c_void_p] * 4
    return lib


def time_reference(lib, n, m, R32, C, E, outdeg, sources, threads, want_dist=False):
    """SSSP from each source by the reference's loop, `threads` sources side
    by side.  Returns (wall seconds, reached edges per source, distances
    n x len(sources) column-major or None)."""
    src = np.ascontiguousarray(sources, dtype=np.uint32)
    k = src.shape[0]
    reached = np.zeros(k, np.uint64)
    secs_each = np.zeros(k, np.float64)
    dist = np.empty((k, n), np.uint32) if want_dist else None
    od = np.ascontiguousarray(outdeg, dtype=np.uint64)
    p = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    with reference_output_silenced():
        secs = lib.ref_sssp_sources(n, m, p(R32), p(C), p(E), p(src), k, threads, p(od),
                                    p(reached), p(secs_each), p(dist))
    if secs < 0:
        raise RuntimeError(f"reference loop failed ({secs})")
    return secs, reached, dist


def ref_sample_text(n, m, k, threads, per_step=1):
    step = "one source per step" if per_step == 1 else f"{per_step} sources per step"
    return (f"SSSP from {k} of the workload's sources on the same R-MAT graph ({n} vertices, "
            f"{m} edges), {step}, by farkhor/KiTES's own kites::sanity_check loop "
            f"(single-threaded per source), {threads} sources side by side on {threads} host "
            f"threads")


def run_reference(args):
    world, rank, _ = dist_setup("gloo")
    if rank != 0:
        return 0
    lib = load_ref_lib()
    if lib is None:
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libref_harness.so not built "
                                         "(needs the reference tree at build time)"}))
        return 0
    n, m, R, C, E, outdeg = make_graph_oracle(args.scale, args.edge_factor, args.seed)
    if int(R[-1]) >= 1 << 31:
        print(json.dumps({"impl": "reference",
                          "unavailable": "the reference loop masks bit 31 of row offsets"}))
        return 0
    R32 = R.astype(np.uint32)
    del R
    threads = host_threads(args.ref_threads)
    # A step is a sample of the workload's sources: one source, or as many as
    # let the K timed steps fill every host thread in one wave.
    per_step = max(1, threads // max(1, args.steps))
    k = args.steps * per_step
    srcs = pick_sources(outdeg, max(args.sources, k + args.warmup), args.seed)
    # Warm-up: W sources side by side, untimed; then exactly K steps, the
    # first K x per_step of the workload's sources, timed from the first
    # loop's start to the last one's end.
    if args.warmup:
        time_reference(lib, n, m, R32, C, E, outdeg, srcs[k:k + args.warmup], threads)
    secs, reached, _ = time_reference(lib, n, m, R32, C, E, outdeg, srcs[:k], threads)
    value = float(reached.sum()) / secs / 1e9
    used = min(threads, k)
    config = dict(workload_config(args), mode="reference CPU loop", batch=1,
                  sources_per_step=per_step, strategy="kites::sanity_check (Gauss-Seidel sweep)",
                  threads=used, batch_gather=None)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "metric_detail": METRIC_DETAIL, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": config,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": used,
                         "kind": "reference",
                         "sample": ref_sample_text(n, m, k, used, per_step)},
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
    if args.batch_selector:
        eng.selector_load_batch(np.fromfile(args.batch_selector, dtype="<f4"))
    g = capi.Graph(eng, R, C, E)
    g.set_batch_gather({"loads": 0, "tma": 1, "async": 2}[args.batch_gather])
    if args.mode == "single" and (args.strategy == "mip" or args.coarse == "mip"):
        g.build_mipmap(args.mip_block)
        if args.coarse == "mip":
            g.set_coarse(capi.STRATEGY_MIP)
    stream = torch.cuda.ExternalStream(g.device_view().stream, device=device)
    srcs = pick_sources(outdeg, args.sources, args.seed, offset=rank)
    K = args.batch
    if args.mode == "batch" and args.sources % K:
        raise SystemExit("--sources must be a multiple of --batch")
    groups = [srcs[i:i + K] for i in range(0, len(srcs), K)]
    if args.mode == "batch" and args.strategy not in ("plain", "auto", "push", "pull_all",
                                                      "pull_changed"):
        raise SystemExit(f"--mode batch does not take --strategy {args.strategy}")
    tuned = None
    if not args.no_autotune:
        r = g.autotune(srcs[:8], batch=K if args.mode == "batch" else 16)
        tuned = {"batch_chunk_items": int(r.batch_chunk_items),
                 "dense_edges": int(r.dense_edges), "dense_rows": int(r.dense_rows),
                 "tpv_strategy": int(r.tpv_strategy), "coarse_strategy": int(r.coarse_strategy),
                 "trials": int(r.trials)}
    loop = 0 if args.host_loop else 1
    bopts = capi.default_opts(device_loop=loop, strategy=STRATEGIES[args.strategy])
    sopts = capi.default_opts(device_loop=loop, strategy=STRATEGIES[args.strategy])
    if args.margin is not None:
        bopts.selector_margin = sopts.selector_margin = args.margin
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

    # The drop-in API with user functions: kites::process with the reference
    # example's four lambdas (examples/sssp_binary_csc.cu, compiled against
    # include/kites/) on the same graph file, a few of the same sources; the
    # last source's distances must equal the engine's (INF 2^30 - 1 there).
    lambda_path = None
    exe = os.path.join(ROOT, "examples", "_build", "sssp_binary_csc")
    if rank == 0 and world == 1 and not args.no_lambda and os.path.exists(exe):
        import tempfile
        lsrc = [int(x) for x in srcs[:args.lambda_sources]]
        with tempfile.TemporaryDirectory() as td:
            dump = os.path.join(td, "V.bin")
            r = subprocess.run([exe, cache_path(args.scale, args.edge_factor, args.seed)] +
                               [str(x) for x in lsrc] + ["--dump", dump],
                               capture_output=True, text=True, timeout=1200)
            if r.returncode != 0:
                raise RuntimeError("sssp_binary_csc failed: " + r.stderr[-500:])
            recs = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
            got = np.fromfile(dump, dtype=np.uint32)[:n]
        ref, _ = g.sssp(lsrc[-1], out=np.empty(n, np.uint32))
        ok = bool(np.array_equal(np.where(got == 1073741823, 0xFFFFFFFF, got), ref))
        lms = sum(x["device_ms"] for x in recs)
        lambda_path = {"value": sum(x["reached_edges"] for x in recs) / (lms * 1e-3) / 1e9,
                       "unit": UNIT, "sources": len(recs), "ms_per_source": lms / len(recs),
                       "iterations": [x["iterations"] for x in recs],
                       "bit_exact_vs_engine": ok,
                       "program": "examples/sssp_binary_csc.cu (kites::process, the reference "
                                  "example's lambdas)"}

    # The fixed batched pull (strategy plain) on the same batches, beside a
    # batched run with another strategy.
    batched_plain = None
    if args.mode == "batch" and args.strategy != "plain":
        fixed = capi.default_opts(device_loop=loop)
        for grp in groups:
            capi._check(lib.kites_sssp_batch(eng._h, g._h, capi.OP_SSSP, capi._p(grp), K, None,
                                             ctypes.byref(fixed), None))
        barrier(world)
        torch.cuda.synchronize()
        q0 = torch.cuda.Event(enable_timing=True)
        q1 = torch.cuda.Event(enable_timing=True)
        q0.record(stream)
        for _ in range(args.steps):
            for grp in groups:
                capi._check(lib.kites_sssp_batch(eng._h, g._h, capi.OP_SSSP, capi._p(grp), K,
                                                 None, ctypes.byref(fixed), None))
        q1.record(stream)
        torch.cuda.synchronize()
        qms = reduce_over_ranks(q0.elapsed_time(q1), world, device, "MAX")
        batched_plain = {"value": total_units / (qms * 1e-3) / 1e9, "unit": UNIT,
                         "ms_per_step": qms / args.steps}

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
    kname = "k_pull_batch_async" if args.batch_gather == "async" else "k_pull_batch"
    prof = os.path.join(ROOT, "profiles", f"{kname}_K{K}_rmat{args.scale}_traffic.md")
    if args.mode == "batch" and os.path.exists(prof):
        import re
        hit = re.search(r"DRAM bytes per launch \(read \+ write, mean\): ([0-9]+)",
                        open(prof).read())
        traffic = int(hit.group(1)) if hit else None
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
        # Each batch's V x K result leaves through kites_sssp_batch_async: its
        # copy to pinned host memory runs under the next batch's compute;
        # the join puts the last copy inside the timed region.  Untimed
        # warm-up calls first (the first one allocates the graph's staging
        # buffer for the asynchronous copies).
        for _ in range(max(1, args.warmup)):
            capi._check(lib.kites_sssp_batch_async(eng._h, g._h, capi.OP_SSSP,
                                                   capi._p(groups[0]), K, capi._p(pinned),
                                                   ctypes.byref(bopts), None))
        capi._check(lib.kites_engine_sync(eng._h))
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        returns = []
        t_host = time.perf_counter()
        e0.record(stream)
        for _ in range(args.steps):
            for grp in groups:
                capi._check(lib.kites_sssp_batch_async(eng._h, g._h, capi.OP_SSSP, capi._p(grp),
                                                       K, capi._p(pinned), ctypes.byref(bopts),
                                                       None))
                returns.append(round((time.perf_counter() - t_host) * 1e3, 2))
        capi._check(lib.kites_engine_join(eng._h))
        e1.record(stream)
        torch.cuda.synchronize()
        e_ms = reduce_over_ranks(e0.elapsed_time(e1), world, device, "MAX")
        # The same device-to-host copy alone, for scale: the pipeline is bound
        # by it whenever it takes longer than a batch's compute.
        src_dev = torch.empty((n, K), dtype=torch.int32, device=device)
        torch.cuda.synchronize()
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record()
        pinned.copy_(src_dev, non_blocking=True)
        c1.record()
        torch.cuda.synchronize()
        d2h_gbs = 4.0 * n * K / (c0.elapsed_time(c1) * 1e-3) / 1e9
        del src_dev
        e2e = {"value": total_units / (e_ms * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": 4 * len(srcs),
               "d2h_bytes_per_step": 4 * n * len(srcs),
               "d2h_gbs_alone": d2h_gbs, "call_returns_ms": returns}

    # Correctness of what was timed, after the timed region: the distances of
    # the first batch (or the first sources of --mode single), column for
    # column bit-exact against the plain single-source kernel, and -- with
    # the CPU baseline -- against farkhor/KiTES's own loop on the same
    # sources, which is also the CPU baseline's timed sample.
    first = groups[0] if args.mode == "batch" else srcs[:K]
    got = np.empty((n, len(first)), np.uint32)
    if args.mode == "batch":
        capi._check(lib.kites_sssp_batch(eng._h, g._h, capi.OP_SSSP, capi._p(first), K,
                                         capi._p(got), ctypes.byref(bopts), None))
    else:
        col = np.empty(n, np.uint32)
        for j, s_ in enumerate(first):
            got[:, j] = g.sssp(int(s_), out=col, opts=sopts)[0]
    plain_cols = [0, len(first) - 1]
    single = np.empty(n, np.uint32)
    ok_plain = all(np.array_equal(got[:, j], g.sssp(int(first[j]), out=single)[0])
                   for j in plain_cols)
    checked = {"columns_vs_plain_kernel": len(plain_cols), "bit_exact_vs_plain": ok_plain}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rlib = load_ref_lib()
        if rlib is not None and int(R[-1]) < 1 << 31:
            threads = host_threads(args.ref_threads)
            k = min(threads, len(first))
            secs, reached_ref, ref_dist = time_reference(
                rlib, n, m, R.astype(np.uint32), C, E, outdeg, first[:k], threads,
                want_dist=True)
            ok_ref = all(np.array_equal(got[:, j], ref_dist[j]) for j in range(k))
            checked.update(columns_vs_reference_loop=k, bit_exact_vs_reference=ok_ref)
            cpu = {"value": float(reached_ref.sum()) / secs / 1e9, "unit": UNIT, "cores": k,
                   "kind": "reference",
                   "sample": ref_sample_text(n, m, k, k) + f" ({secs:.1f} s)"}
    checked["ok"] = all(v for key, v in checked.items() if key.startswith("bit_exact"))
    del got

    if rank == 0:
        line = {
            "metric": METRIC, "metric_detail": METRIC_DETAIL, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": dict(workload_config(args), autotuned=tuned),
            "clocks": clk.summary(),
            "e2e": e2e,
            "gpu_launches": int(launches),
            "plain": plain,
            "speedup_vs_plain": (value / plain["value"]) if plain else None,
            "batched_plain": batched_plain,
            "lambda_path": lambda_path,
            "speedup_vs_batched_plain": (value / batched_plain["value"]) if batched_plain
            else None,
            "roofline": ({"bound": "hbm", "achieved": b_ach, "peak": peak, "unit": "GB/s",
                          "frac": b_ach / peak, "traffic": traffic,
                          "kernel": (f"k_pull_batch_async<SSSP,K={K}>" if args.batch_gather == "async"
                                     else f"k_pull_batch<SSSP,K={K}>"),
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
            "checked": checked,
        }
        print(json.dumps(line))
    g.close()
    eng.close()
    if world > 1:
        import torch.distributed as tdist
        tdist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# the other configurations (--suite)
# ---------------------------------------------------------------------------

def run_suite(args):
    """One line per configuration, each timed on the device (CUDA events of
    the engine, device loop) after one untimed run; results are checked
    against a second strategy or the plain kernel where one exists."""
    from kites_b200 import capi

    eng = capi.Engine(0)
    lines = []

    def emit(workload, value, unit, **kw):
        rec = {"suite": True, "workload": workload, "value": value, "unit": unit, **kw}
        lines.append(rec)
        print(json.dumps(rec), flush=True)

    def timed(fn, reps):
        fn()
        return min(fn() for _ in range(reps))

    # Config 1: 7,115 vertices, 103,689 edges, SSSP from vertex 0 through
    # kites_process (the reference's process() call), weights U[1,63].
    s, d, w = capi.gen_rmat(13, 103689, seed=1, w_lo=1, w_hi=63, n_vertices=7115)
    R, C, E = capi.csc_from_edges(7115, s, d, w)
    g = capi.Graph(eng, R, C, E)
    outdeg = np.bincount(C, minlength=7115).astype(np.uint64)
    dist, _ = g.sssp(0)
    reach = reached_edges(dist, outdeg)
    for loop in (1, 0):
        ms = timed(lambda: g.sssp(0, out=False, opts=capi.default_opts(device_loop=loop))[1]
                   .device_ms, 20)
        emit("cfg1_sssp", reach / (ms * 1e-3) / 1e9, UNIT, ms=ms,
             loop="device (CUDA graph)" if loop else "host (flag read back per iteration)")
    g.close()

    # Scale 22, R-MAT and Erdos-Renyi: plain SSSP and BFS from 8 sources,
    # min-label CC on the symmetrised graph.
    n = 1 << 22
    for kind in ("rmat22", "er22"):
        if kind == "rmat22":
            s, d, w = capi.gen_rmat(22, 16 * n, seed=1)
        else:
            s, d, w = capi.gen_er(n, 16 * n, seed=1)
        R, C, E = capi.csc_from_edges(n, s, d, w)
        g = capi.Graph(eng, R, C, E)
        outdeg = np.bincount(C, minlength=n).astype(np.uint64)
        srcs = pick_sources(outdeg, 8, args.seed)
        for op, name in ((capi.OP_SSSP, "sssp"), (capi.OP_BFS, "bfs")):
            for strat, sname in ((capi.STRATEGY_PLAIN, "plain"), (capi.STRATEGY_AUTO, "auto")):
                o = capi.default_opts(strategy=strat)
                tot_ms, tot_e = 0.0, 0
                for src in srcs:
                    dist, st = g.sssp(int(src), op=op, opts=o)
                    tot_ms += timed(lambda: g.sssp(int(src), op=op, out=False, opts=o)[1]
                                    .device_ms, 2)
                    tot_e += reached_edges(dist, outdeg)
                emit(f"{kind}_{name}", tot_e / (tot_ms * 1e-3) / 1e9, UNIT, sources=len(srcs),
                     strategy=sname, ms_per_source=tot_ms / len(srcs))
        g.close()
        # Both directions of every edge as a directed graph (the per-iteration
        # strategies take directed graphs; the labels are those of the
        # undirected graph).
        gs = capi.Graph.from_edges(eng, n, np.concatenate([s, d]), np.concatenate([d, s]),
                                   directed=True)
        want = None
        for strat, sname in ((capi.STRATEGY_PLAIN, "plain"), (capi.STRATEGY_PUSH, "push"),
                             (capi.STRATEGY_AUTO, "auto")):
            o = capi.default_opts(strategy=strat)
            labels, _ = gs.cc(opts=o)
            if want is None:
                want = labels.copy()
            ms = timed(lambda: gs.cc(opts=o)[1].device_ms, 2)
            emit(f"{kind}_cc", 2 * s.shape[0] / (ms * 1e-3) / 1e9, "GTEPS (edges of the "
                 "symmetrised graph per run)", ms=ms, strategy=sname,
                 bit_exact_vs_plain=bool(np.array_equal(labels, want)))
        gs.close()
        del s, d, w, R, C, E

    # A 2048 x 2048 grid (road-like, weights U[1, 1000]): plain, AUTO, the
    # mipmapped frontier (blocks of one grid row) alone and as AUTO's coarse
    # class, 4 sources each, distances checked against plain.
    side = 2048
    n = side * side
    s, d, w = capi.gen_grid(side, seed=1, w_lo=1, w_hi=1000)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(eng, R, C, E)
    g.build_mipmap(side)
    outdeg = np.bincount(C, minlength=n).astype(np.uint64)
    srcs = pick_sources(outdeg, 4, args.seed)
    want = {}
    for strat, coarse, sname in ((capi.STRATEGY_PLAIN, None, "plain"),
                                 (capi.STRATEGY_AUTO, capi.STRATEGY_PULL_ALL, "auto"),
                                 (capi.STRATEGY_MIP, None, "mip"),
                                 (capi.STRATEGY_AUTO, capi.STRATEGY_MIP, "auto_coarse_mip")):
        if coarse is not None:
            g.set_coarse(coarse)
        o = capi.default_opts(strategy=strat)
        tot_ms, tot_e, ok = 0.0, 0, True
        for src in srcs:
            dist, st = g.sssp(int(src), opts=o)
            if sname == "plain":
                want[int(src)] = dist.copy()
            ok = ok and bool(np.array_equal(dist, want[int(src)]))
            tot_ms += timed(lambda: g.sssp(int(src), out=False, opts=o)[1].device_ms, 2)
            tot_e += reached_edges(dist, outdeg)
        emit("grid2048_sssp", tot_e / (tot_ms * 1e-3) / 1e9, UNIT, sources=len(srcs),
             strategy=sname, ms_per_source=tot_ms / len(srcs), bit_exact_vs_plain=ok,
             block_vertices=side)
    g.set_coarse(capi.STRATEGY_PULL_ALL)
    g.close()
    del s, d, w, R, C, E

    # 256 seeded sources on R-MAT scale 20 as one K = 256 batch.
    n = 1 << 20
    s, d, w = capi.gen_rmat(20, 16 * n, seed=1)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    g = capi.Graph(eng, R, C, E)
    outdeg = np.bincount(C, minlength=n).astype(np.uint64)
    srcs = pick_sources(outdeg, 256, args.seed)
    out = np.empty((n, 256), np.uint32)
    want = None
    for strat, sname in ((capi.STRATEGY_PLAIN, "plain"), (capi.STRATEGY_AUTO, "auto")):
        o = capi.default_opts(strategy=strat)
        g.sssp_batch(srcs, out=out, opts=o)
        if want is None:
            want = out.copy()
            reach = sum(reached_edges(want[:, j], outdeg) for j in range(256))
        ok = bool(np.array_equal(out, want))
        ms = timed(lambda: g.sssp_batch(srcs, out=out, opts=o)[1].device_ms, 2)
        emit("rmat20_batch256", reach / (ms * 1e-3) / 1e9, UNIT, ms=ms, strategy=sname,
             bit_exact_vs_plain=ok)
    # PageRank, 20 iterations (GTEPS = 20 m / time).
    ms = timed(lambda: g.pagerank(iterations=20)[1].device_ms, 2)
    emit("rmat20_pagerank20", 20 * C.shape[0] / (ms * 1e-3) / 1e9, "GTEPS (20 m per run)",
         ms=ms)
    g.close()
    del s, d, w, R, C, E, out, want

    # 1,000 R-MAT graphs (vertices log-uniform in [1K, 100K], edge factor
    # U[4, 32]) as one disjoint union, one seed (vertex 0 of each) per graph,
    # one device loop.
    s, d, w, vo, eo = capi.gen_rmat_union(1000, seed=1)
    nn = int(vo[-1])
    R, C, E = capi.csc_from_edges(nn, s, d, w)
    g = capi.Graph(eng, R, C, E)
    seeds = vo[:-1].astype(np.uint32)
    dist, _ = g.sssp_multi_seed(seeds)
    outdeg = np.bincount(C, minlength=nn).astype(np.uint64)
    reach = reached_edges(dist, outdeg)
    ms = timed(lambda: g.sssp_multi_seed(seeds, out=False)[1].device_ms, 3)
    emit("multigraph1000_sssp", reach / (ms * 1e-3) / 1e9, UNIT, ms=ms, graphs=1000,
         vertices=nn, edges=int(eo[-1]))
    g.close()
    eng.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.suite:
        return run_suite(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
