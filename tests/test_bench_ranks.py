"""bench.py's multi-rank plumbing on CPU: two gloo ranks agree on the max of
their timings, pass the barrier, and the reference arm prints from rank 0
only (the path a torchrun launch of bench.py takes, without GPUs)."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world, cuda=False)
        t = bench.max_over_ranks(1.0 + rank, world, device="cpu")
        out.put((rank, t))
        bench.barrier(world, cuda=False)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_barrier_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res == {0: 2.0, 1: 2.0}


def test_reference_arm_prints_from_rank0_only():
    def run(rank):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank))
        return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "16",
                               "--steps", "1", "--warmup", "1", "--gpus", "2"],
                              capture_output=True, text=True, env=env, timeout=300)
    r1 = run(1)
    assert r1.returncode == 0 and r1.stdout.strip() == ""
    r0 = run(0)
    assert r0.returncode == 0
    line = json.loads(r0.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
