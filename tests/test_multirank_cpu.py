"""The multi-GPU bench path is replicas: every rank times its own contractions and rank 0
reports the slowest rank's time and the whole-job throughput. Its host logic runs here as two
gloo ranks on CPU (127.0.0.1): both ranks see the maximum, the value counts every rank's
work, and the reference arm prints only on rank 0."""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path[:0] = [ROOT]
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks(10.0 + 5.0 * rank, "cpu", world)
        q.put((rank, got, bench.whole_job_value(1e9, world, 4, got)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_value_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [15.0, 15.0]
    # 2 ranks × 4 steps × 1 GFLOP in 15 ms
    assert all(abs(r[2] - 2 * 4 * 1e9 / 15e-3 / 1e9) < 1e-9 for r in res)


def test_reference_arm_prints_only_on_rank0():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", "u1_small", "--steps", "1", "--warmup", "1", "--gpus", "2"],
                         env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == ""
    env0 = dict(env, RANK="0", LOCAL_RANK="0")
    out0 = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                           "--workload", "u1_small", "--steps", "1", "--warmup", "1", "--gpus", "2"],
                          env=env0, capture_output=True, text=True, timeout=300)
    assert out0.returncode == 0
    line = json.loads(out0.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
