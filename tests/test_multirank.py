"""Multi-rank host logic on CPU (gloo, world size 2): the benchmark's
max-over-ranks timing, the sharding of the serving stream across replicas,
and the reference arm under torchrun (rank 0 alone measures and prints)."""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _reduce_worker(rank, world, port, q):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q.put((rank, bench.reduce_max(1.5 + 10.0 * rank, dist, "cpu")))
    finally:
        dist.destroy_process_group()


def test_reduce_max_over_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29400 + os.getpid() % 500
    procs = [ctx.Process(target=_reduce_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 11.5, 1: 11.5}


def test_reduce_max_single_process():
    import bench
    assert bench.reduce_max(3.25, None, "cpu") == 3.25


def test_serving_shards_partition_the_stream(b200):
    import importlib
    import bench
    srv = importlib.import_module("hiflow3_b200.serving")
    stream = srv.c5_stream(1000, seed=4)
    for world in (1, 2, 3, 8):
        parts = [bench.shard(stream, r, world) for r in range(world)]
        assert sum(len(p) for p in parts) == len(stream)
        seeds = sorted(x["rhs_seed"] for p in parts for x in p)
        assert seeds == sorted(x["rhs_seed"] for x in stream)
        assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1


def test_reference_arm_under_torchrun():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libhiflow_lmp_ref.so")):
        pytest.skip("reference CPU library (oracle/_ref) not built")
    port = 29900 + os.getpid() % 90
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--N", "12"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["value"] > 0
    assert rec["cpu_baseline"]["kind"] == "reference" and rec["cpu_baseline"]["cores"] >= 1
    assert rec["e2e"]["h2d_bytes_per_step"] == 0
    # the arm runs the reference's own code only: no library of this platform
    assert rec["libraries_loaded"] == ["oracle/_ref/libhiflow_lmp_ref.so"], rec["libraries_loaded"]
    assert rec["solve"]["relres_true"] <= 1e-10
