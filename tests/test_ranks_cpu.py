"""Multi-rank (replica) logic of bench.py on CPU: two gloo ranks.

The dycore does not shard, so N GPUs run N independent replicas; the only
cross-rank operations are the barrier and the max over ranks of the timed
region.  These tests run that logic with world_size 2 over gloo, and the
reference arm under torchrun, where rank 0 alone measures and prints.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        # rank r pretends its timed region took (r + 1) * 10 ms
        ms = bench.max_over_ranks(10.0 * (rank + 1), world, "cpu")
        value = bench.replica_throughput(world, 1000, 5, ms * 1e-3)
        q.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, ms, value in got:
        assert ms == 20.0                       # the slowest rank's time
        assert value == pytest.approx(2 * 1000 * 5 / 0.020)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.replica_throughput(1, 100, 2, 0.5) == 400.0


def test_reference_arm_under_torchrun_world2():
    """bench.py --impl reference with 2 ranks: rank 0 prints one JSON line,
    rank 1 exits 0 without work."""
    port = _free_port()
    env = dict(os.environ, OMP_NUM_THREADS="4")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--case", "abl_dry", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "cell-RK3-steps/s" and d["n_gpus"] == 2
    assert d["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port"
