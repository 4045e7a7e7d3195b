"""Trains the learned per-iteration strategy selector on generated graphs.

    python -m kites_b200.train_selector [--out PATH] [--inc PATH] [--quick]
                                        [--eval-scale S] [--eval-sources K]

Training set (seeded, generated on the host):
  * R-MAT graphs of scales 16-22, edge factor 8-32, (a, b, c) jittered
    around (0.57, 0.19, 0.19), weights U[1, 255];
  * Erdos-Renyi graphs with 2^16 - 2^21 vertices, edge factor 4-16;
  * 2-D grids of side 256-1536 (4-neighbour, weights U[1, 1000]).
For each graph, a few seeded sources with out-edges run through
kites_selector_record: at every iteration each selector class (PLAIN, PUSH,
PULL_ALL, the graph's TPV width) runs from the same state and is timed.
The MLP (12 -> 32 -> 32 -> 4, FP32) is trained on the device with
kites_selector_train (full-batch Adam on the log time ratios), each
iteration repeated in proportion to its PLAIN time (1 to 16 times) so that
the fit follows the iterations a run's time is made of.  --config3 N trains
on N graphs of the selector configuration's recipe instead (four in five
R-MAT graphs of scales 16-22 with jittered a, b, c; one in five grids of
side 1024-4096).

Held-out evaluation: SSSP from --eval-sources seeded sources on R-MAT scale
--eval-scale (the benchmark graph's generator and parameters, a different
seed), AUTO against PLAIN, both through the CUDA-graph device loop, plus the
"oracle-best" schedule (the per-iteration minimum over the recorded class
times of one source) as the ceiling.

Outputs: the 1628 parameters as raw little-endian float32 (--out) and as a
C initialiser (--inc) that the library compiles in as its default selector.

--batch K trains the batched loop's selector instead (classes PLAIN, PUSH,
PULL_ALL, PULL_CHANGED of kites_sssp_batch): the same graphs, K seeded
sources per recorded run (kites_selector_record_batch), fitted with
kites_selector_fit and written for selector_batch_default.inc; the held-out
evaluation runs K-source batches of batched AUTO against batched PLAIN.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

from kites_b200 import capi

HERE = os.path.dirname(os.path.abspath(__file__))


def splitmix(seed: int, k: int) -> int:
    mask = (1 << 64) - 1
    z = (seed * 0x9E3779B97F4A7C15 + (k + 1) * 0xBF58476D1CE4E5B9) & mask
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
    return z ^ (z >> 31)


def uniform(seed: int, k: int, lo: float, hi: float) -> float:
    return lo + (hi - lo) * (splitmix(seed, k) >> 11) / float(1 << 53)


def config3_specs(n_graphs: int = 200):
    """The selector training set of the benchmark configuration: n_graphs
    seeded graphs, four in five R-MAT (scale uniform in 16..22, edge factor
    16, (a, b, c) uniform within +-0.04 of (0.57, 0.19, 0.19), scaled down to
    a sum of 0.99 where they pass it), one in five a 2-D grid road-like graph
    (side log-uniform in 1024..4096, 4-neighbour, weights U[1, 1000])."""
    specs = []
    for i in range(n_graphs):
        seed = 5000 + i
        if i % 5 == 4:
            side = int(round(1024 * 4 ** uniform(seed, 0, 0.0, 1.0)))
            specs.append(("grid", side, 4, 0, 0, 0, seed))
            continue
        sc = 16 + int(uniform(seed, 0, 0, 7))
        a = uniform(seed, 1, 0.53, 0.61)
        b = uniform(seed, 2, 0.15, 0.23)
        c = uniform(seed, 3, 0.15, 0.23)
        if a + b + c > 0.99:
            f = 0.99 / (a + b + c)
            a, b, c = a * f, b * f, c * f
        specs.append(("rmat", sc, 16, a, b, c, seed))
    return specs


def training_graphs(quick: bool, config3: int = 0):
    """(name, n, src, dst, w) tuples, generated one at a time."""
    specs = []
    scales = [16, 17, 18, 19, 20, 21, 22] if not quick else [16, 18, 20]
    for i, sc in enumerate(scales):
        for j in range(3 if not quick else 1):
            seed = 1000 + 10 * i + j
            a = uniform(seed, 0, 0.45, 0.65)
            b = uniform(seed, 1, 0.12, 0.25)
            c = uniform(seed, 2, 0.12, 0.25)
            if a + b + c > 0.97:
                c = 0.97 - a - b
            ef = int(uniform(seed, 3, 8, 32))
            specs.append(("rmat", sc, ef, a, b, c, seed))
    for i, lv in enumerate([16, 18, 20, 21] if not quick else [16, 19]):
        seed = 2000 + i
        specs.append(("er", lv, int(uniform(seed, 0, 4, 16)), 0, 0, 0, seed))
    for i, side in enumerate([256, 512, 1024, 1536] if not quick else [256, 768]):
        specs.append(("grid", side, 4, 0, 0, 0, 3000 + i))
    if config3:
        specs = config3_specs(config3)
    for kind, p, ef, a, b, c, seed in specs:
        if kind == "rmat":
            n = 1 << p
            s, d, w = capi.gen_rmat(p, ef * n, a, b, c, seed, 1, 255)
            name = f"rmat{p}_ef{ef}_a{a:.2f}b{b:.2f}c{c:.2f}"
        elif kind == "er":
            n = 1 << p
            s, d, w = capi.gen_er(n, ef * n, seed, 1, 255)
            name = f"er{p}_ef{ef}"
        else:
            n = p * p
            s, d, w = capi.gen_grid(p, seed, 1, 1000)
            name = f"grid{p}"
        yield name, n, s, d, w, seed


def pick_sources(src, n, count, seed):
    deg = np.bincount(src, minlength=n)
    cand = np.flatnonzero(deg > 0)
    return [int(cand[splitmix(seed, 7 + k) % cand.shape[0]]) for k in range(count)]


def collect(eng, quick: bool, per_graph: int, log, config3: int = 0):
    Xs, Ts = [], []
    for name, n, s, d, w, seed in training_graphs(quick, config3):
        t0 = time.time()
        R, C, E = capi.csc_from_edges(n, s, d, w)
        srcs = pick_sources(s, n, per_graph, seed)
        del s, d, w
        g = capi.Graph(eng, R, C, E)
        rows = 0
        cap = 32768 if name.startswith("grid") else 1024
        for src in srcs:
            X, T = g.selector_record(capi.OP_SSSP, src, capacity=cap)
            Xs.append(X)
            Ts.append(T)
            rows += X.shape[0]
        g.close()
        log(f"{name}: {rows} iterations from {len(srcs)} sources in {time.time() - t0:.1f}s")
    return np.concatenate(Xs), np.concatenate(Ts)


def batch_training_graphs(quick: bool):
    """The batched selector's training graphs: R-MAT scales 18-24 (two per
    scale, a, b, c jittered as config3_specs does; seeds other than the
    evaluation graph's), Erdos-Renyi graphs of 2^20 and 2^22 vertices and two
    grids.  The batched classes trade gathers against atomics whose cost
    depends on whether the V x K array fits in L2, so the scales reach the
    benchmark's."""
    specs = []
    scales = [18, 20, 22, 24] if quick else [18, 19, 20, 21, 22, 23, 24]
    for sc in scales:
        for j in range(1 if quick else 2):
            seed = 7000 + 10 * sc + j
            a = uniform(seed, 1, 0.53, 0.61)
            b = uniform(seed, 2, 0.15, 0.23)
            c = uniform(seed, 3, 0.15, 0.23)
            if a + b + c > 0.99:
                f = 0.99 / (a + b + c)
                a, b, c = a * f, b * f, c * f
            specs.append(("rmat", sc, 16, a, b, c, seed))
    for lv in ([20] if quick else [20, 22]):
        specs.append(("er", lv, 16, 0, 0, 0, 7500 + lv))
    for side in ([512] if quick else [512, 1024]):
        specs.append(("grid", side, 4, 0, 0, 0, 7600 + side))
    for kind, p, ef, a, b, c, seed in specs:
        if kind == "rmat":
            n = 1 << p
            s, d, w = capi.gen_rmat(p, ef * n, a, b, c, seed, 1, 255)
            name = f"rmat{p}_a{a:.2f}b{b:.2f}c{c:.2f}"
        elif kind == "er":
            n = 1 << p
            s, d, w = capi.gen_er(n, ef * n, seed, 1, 255)
            name = f"er{p}"
        else:
            n = p * p
            s, d, w = capi.gen_grid(p, seed, 1, 1000)
            name = f"grid{p}"
        yield name, n, s, d, w, seed


def time_weighted(X, T, cap=16):
    """Repeats each iteration in proportion to its PLAIN time (at least once,
    at most `cap` times), so that the fit follows the iterations that make
    up a run's time, not the many short ones."""
    w = T[:, 0] / max(float(np.median(T[:, 0])), 1e-3)
    reps = np.clip(np.rint(w), 1, cap).astype(np.int64)
    return np.repeat(X, reps, axis=0), np.repeat(T, reps, axis=0)


def collect_batch(eng, quick: bool, k: int, runs: int, log, config3: int = 0):
    Xs, Ts = [], []
    graphs = training_graphs(quick, config3) if config3 else batch_training_graphs(quick)
    for name, n, s, d, w, seed in graphs:
        t0 = time.time()
        R, C, E = capi.csc_from_edges(n, s, d, w)
        del s, d, w
        outdeg = np.bincount(C, minlength=n)
        cand = np.flatnonzero(outdeg > 0)
        g = capi.Graph(eng, R, C, E)
        rows = 0
        cap = 32768 if name.startswith("grid") else 1024
        for r in range(runs):
            srcs = np.array([cand[splitmix(seed, 100 * r + j) % cand.shape[0]]
                             for j in range(k)], dtype=np.uint32)
            X, T = g.selector_record_batch(srcs, capi.OP_SSSP, capacity=cap)
            Xs.append(X)
            Ts.append(T)
            rows += X.shape[0]
        g.close()
        log(f"{name}: {rows} batched iterations from {runs} runs of {k} in "
            f"{time.time() - t0:.1f}s")
    return np.concatenate(Xs), np.concatenate(Ts)


def evaluate_batch(eng, scale: int, k: int, batches: int, seed: int, log):
    n = 1 << scale
    s, d, w = capi.gen_rmat(scale, 16 * n, 0.57, 0.19, 0.19, seed, 1, 255)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    del s, d, w
    outdeg = np.bincount(C, minlength=n)
    cand = np.flatnonzero(outdeg > 0)
    g = capi.Graph(eng, R, C, E)
    del C, E
    groups = [np.array([cand[splitmix(seed, 1000 * b + j) % cand.shape[0]] for j in range(k)],
                       dtype=np.uint32) for b in range(batches)]
    res, want = {}, {}
    out = np.empty((n, k), np.uint32)
    for name, strat in (("plain", capi.STRATEGY_PLAIN), ("auto", capi.STRATEGY_AUTO),
                        ("push", capi.STRATEGY_PUSH), ("pull_all", capi.STRATEGY_PULL_ALL),
                        ("pull_changed", capi.STRATEGY_PULL_CHANGED)):
        o = capi.default_opts(strategy=strat)
        g.sssp_batch(groups[0], out=out, opts=o)  # warm-up (captures the device loop)
        total, hist = 0.0, np.zeros(capi.STRATEGY_COUNT, np.uint64)
        for b, grp in enumerate(groups):
            _, st = g.sssp_batch(grp, out=out, opts=o)
            digest = hashlib.blake2b(memoryview(out).cast("B"), digest_size=16).digest()
            if name == "plain":
                want[b] = digest
            elif digest != want[b]:
                raise RuntimeError(f"batched {name} differs from batched plain on batch {b}")
            total += st.device_ms
            hist += np.array(st.strategy_hist[:], dtype=np.uint64)
        res[name] = {"device_ms": total, "strategy_hist": hist.tolist()}
        log(f"eval batched {name}: {total:.2f} ms over {batches} batches of {k}")
    # The ceiling on this graph: every class timed at every iteration of the
    # plain trajectory of the first batch.
    X, T = g.selector_record_batch(groups[0], capacity=256)
    res["record_batch0"] = {"iterations": int(X.shape[0]), "class_sum_ms": T.sum(0).tolist(),
                            "oracle_best_ms": float(T.min(1).sum()),
                            "per_iteration_ms": T.tolist()}
    g.close()
    res["auto_speedup_vs_plain"] = res["plain"]["device_ms"] / res["auto"]["device_ms"]
    return res


def validate_batch(eng, scale: int, k: int, batches: int, seed: int, candidates, log):
    """AUTO device time of each candidate parameter set on a validation graph
    (the benchmark's generator with its own seed, distinct from the
    evaluation graph's); returns the index of the fastest."""
    n = 1 << scale
    s, d, w = capi.gen_rmat(scale, 16 * n, 0.57, 0.19, 0.19, seed, 1, 255)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    del s, d, w
    outdeg = np.bincount(C, minlength=n)
    cand = np.flatnonzero(outdeg > 0)
    g = capi.Graph(eng, R, C, E)
    del C, E
    groups = [np.array([cand[splitmix(seed, 1000 * b + j) % cand.shape[0]] for j in range(k)],
                       dtype=np.uint32) for b in range(batches)]
    out = np.empty((n, k), np.uint32)
    o = capi.default_opts(strategy=capi.STRATEGY_AUTO)
    times = []
    for i, params in enumerate(candidates):
        eng.selector_load_batch(params)
        g.sssp_batch(groups[0], out=out, opts=o)  # warm-up
        total = 0.0
        for grp in groups:
            total += g.sssp_batch(grp, out=out, opts=o)[1].device_ms
        times.append(total)
        log(f"validation fit {i}: AUTO {total:.2f} ms over {batches} batches")
    g.close()
    return int(np.argmin(times)), times


def evaluate(eng, scale: int, n_src: int, seed: int, log):
    n = 1 << scale
    s, d, w = capi.gen_rmat(scale, 16 * n, 0.57, 0.19, 0.19, seed, 1, 255)
    R, C, E = capi.csc_from_edges(n, s, d, w)
    srcs = pick_sources(s, n, n_src, seed)
    del s, d, w
    g = capi.Graph(eng, R, C, E)
    res = {}
    want = {}
    for name, strat in (("plain", capi.STRATEGY_PLAIN), ("auto", capi.STRATEGY_AUTO),
                        ("push", capi.STRATEGY_PUSH), ("pull_all", capi.STRATEGY_PULL_ALL)):
        o = capi.default_opts(strategy=strat)
        for src in srcs[:2]:  # warm-up (captures the device loop)
            g.sssp(src, out=False, opts=o)
        total, hist = 0.0, np.zeros(capi.STRATEGY_COUNT, np.uint64)
        for src in srcs:
            dist, st = g.sssp(src, opts=o)
            if name == "plain":
                want[src] = dist.copy()
            elif not np.array_equal(dist, want[src]):
                raise RuntimeError(f"{name} differs from plain on source {src}")
            total += st.device_ms
            hist += np.array(st.strategy_hist[:], dtype=np.uint64)
        res[name] = {"device_ms": total, "strategy_hist": hist.tolist()}
        log(f"eval {name}: {total:.2f} ms over {len(srcs)} sources")
    X, T = g.selector_record(capi.OP_SSSP, srcs[0], capacity=1024)
    res["record_source0"] = {"iterations": int(X.shape[0]),
                             "class_sum_ms": T.sum(0).tolist(),
                             "oracle_best_ms": float(T.min(1).sum())}
    g.close()
    res["auto_speedup_vs_plain"] = res["plain"]["device_ms"] / res["auto"]["device_ms"]
    return res


def write_inc(params: np.ndarray, path: str, meta: str):
    lines = [f"// Default selector parameters ({params.shape[0]} float32), written by",
             "// python -m kites_b200.train_selector.  " + meta]
    body = ",\n".join(", ".join(f"{float(v):.9e}f" for v in params[i:i + 6])
                      for i in range(0, params.shape[0], 6))
    lines.append(body)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "selector_params.f32"))
    ap.add_argument("--inc", default=None, help="also write a C initialiser here")
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--sources-per-graph", type=int, default=3)
    ap.add_argument("--epochs", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--eval-scale", type=int, default=24)
    ap.add_argument("--eval-sources", type=int, default=8)
    ap.add_argument("--eval-seed", type=int, default=99)
    ap.add_argument("--report", default=None, help="write the JSON report here")
    ap.add_argument("--batch", type=int, default=0,
                    help="train the batched selector with batches of this many sources")
    ap.add_argument("--runs-per-graph", type=int, default=2)
    ap.add_argument("--config3", type=int, default=0,
                    help="train on this many graphs of the configuration's recipe "
                         "(R-MAT 16-22 with jittered a,b,c and grids of side 1024-4096)")
    ap.add_argument("--eval-batches", type=int, default=2)
    ap.add_argument("--fits", type=int, default=1,
                    help="batched: fit this many seeds and keep the one whose AUTO is "
                         "fastest on a validation graph (seed --eval-seed + 1)")
    ap.add_argument("--valid-scale", type=int, default=23)
    a = ap.parse_args(argv)

    def log(msg):
        print(msg, flush=True)

    eng = capi.Engine(0)
    t0 = time.time()
    if a.batch:
        X, T = collect_batch(eng, a.quick, a.batch, a.runs_per_graph, log, a.config3)
        T = np.maximum(T, 1e-3)
        log(f"dataset: {X.shape[0]} batched iterations in {time.time() - t0:.1f}s")
        Xw, Tw = time_weighted(X, T)
        fits = [eng.selector_fit(Xw, Tw, epochs=a.epochs, lr=a.lr, seed=1 + i)
                for i in range(max(1, a.fits))]
        best, val_ms = 0, None
        if len(fits) > 1:
            best, val_ms = validate_batch(eng, a.valid_scale, a.batch, a.eval_batches,
                                          a.eval_seed + 1, [p for p, _ in fits], log)
        params, loss = fits[best]
        log(f"trained: loss {loss:.4f} (fit {best} of {len(fits)})")
        eng.selector_load_batch(params)
        params.astype("<f4").tofile(a.out)
        report = {"dataset_iterations": int(X.shape[0]), "weighted_rows": int(Xw.shape[0]),
                  "train_loss": loss, "batch": a.batch, "fits": len(fits), "chosen_fit": best,
                  "validation_auto_ms": val_ms,
                  "class_sum_ms_train": T.sum(0).tolist(),
                  "oracle_best_over_plain_train": float(T[:, 0].sum() / T.min(1).sum())}
        if a.eval_scale:
            report["eval"] = evaluate_batch(eng, a.eval_scale, a.batch, a.eval_batches,
                                            a.eval_seed, log)
        if a.inc:
            write_inc(params, a.inc, f"batched classes, K = {a.batch}, dataset "
                      f"{X.shape[0]} iterations, loss {loss:.4f}")
        log(json.dumps(report))
        if a.report:
            with open(a.report, "w") as f:
                json.dump(report, f, indent=1)
        eng.close()
        return 0
    X, T = collect(eng, a.quick, a.sources_per_graph, log, a.config3)
    T = np.maximum(T, 1e-3)
    log(f"dataset: {X.shape[0]} iterations in {time.time() - t0:.1f}s")
    Xw, Tw = time_weighted(X, T)
    params, loss = eng.selector_train(Xw, Tw, epochs=a.epochs, lr=a.lr, seed=1)
    log(f"trained: loss {loss:.4f}")
    eng.selector_load(params)
    params.astype("<f4").tofile(a.out)
    report = {"dataset_iterations": int(X.shape[0]), "train_loss": loss,
              "oracle_best_over_plain_train": float(T[:, 0].sum() / T.min(1).sum())}
    if a.eval_scale:
        report["eval"] = evaluate(eng, a.eval_scale, a.eval_sources, a.eval_seed, log)
    if a.inc:
        write_inc(params, a.inc, f"dataset {X.shape[0]} iterations, loss {loss:.4f}")
    log(json.dumps(report))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)
    eng.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
