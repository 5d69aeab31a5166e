"""Multi-process plumbing of bench.py on the CPU (gloo, world size 2): the rank setup,
the max-over-ranks timing reduction and the barrier that bracket the timed region, and
the reference arm under torchrun (rank 0 alone works and prints one line)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup(type("A", (), {})())
    bench.barrier(w)
    t = bench.dist_max(1.0 + 2.0 * r, w)       # rank 1 is the slow one
    bench.barrier(w)
    q.put((r, w, t))
    dist.destroy_process_group()


def test_dist_max_and_barrier_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 2, 3.0), (1, 2, 3.0)]


def test_reference_arm_under_torchrun():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "1",
           "--elements", "20000", "--cpu-seconds", "0.5"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["steps"] == 2
    assert d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"
    # the whole workload (the structured mesh rounds 20000 up to whole rows), not a sample
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and 20000 <= d["config"]["elements"] < 20400
    assert d["config"]["updates_per_step"] > 0 and d["ms_per_step"] > 0
