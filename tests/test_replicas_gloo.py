"""Multi-process (replica) logic of bench.py on CPU ranks over gloo.

The path does not shard: N GPUs run N independent replicas, and
torch.distributed only carries the barrier and the max / sum over ranks of
the timings and units.  These tests run that host logic with world_size 2
(rendezvous on 127.0.0.1) and the reference arm under torchrun, where rank 0
alone prints the JSON line."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import numpy as np
    import torch

    import bench
    w, r, _ = bench.dist_setup("gloo")
    assert (w, r) == (world, rank)
    dev = torch.device("cpu")
    mx = bench.reduce_over_ranks(10.0 + rank, w, dev, "MAX")
    sm = bench.reduce_over_ranks(100.0 * (rank + 1), w, dev, "SUM")
    bench.barrier(w)
    outdeg = np.ones(1000, np.uint64)
    srcs = bench.pick_sources(outdeg, 8, 1, offset=rank)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"max": mx, "sum": sm, "srcs": srcs.tolist()}, f)
    import torch.distributed as tdist
    tdist.destroy_process_group()


def test_reductions_and_disjoint_sources_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    for r in res:
        assert r["max"] == 11.0          # max over ranks of the device times
        assert r["sum"] == 300.0         # units of all ranks
    # Each replica draws its own sources (weak scaling: no overlap needed,
    # but the draws differ per rank).
    assert res[0]["srcs"] != res[1]["srcs"]


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_harness.so")),
                    reason="reference harness not built")
def test_reference_arm_under_torchrun_prints_once(tmp_path):
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "2", "--warmup", "1", "--scale", "12"]
    env = dict(os.environ, KITES_GRAPH_CACHE=str(tmp_path))
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["value"] > 0 and rec["n_gpus"] == 2
    assert rec["e2e"]["h2d_bytes_per_step"] == 0
    assert rec["config"]["workload"] == "sssp_rmat_scale12" and rec["cpu_baseline"]["cores"] >= 1
    # The reference process wrote the graph through the oracle alone.
    assert os.listdir(tmp_path) == ["rmat12_ef16_seed1.csc"]
