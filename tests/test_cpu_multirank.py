"""The bench's N > 1 host logic on CPU: two gloo ranks agree on the slowest
rank's time and the whole-job rate; the reference arm prints only on rank 0."""
import os
import subprocess
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, ms, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sys.path.insert(0, ROOT)
        import bench
        value, ms_max = bench.job_rate(ms[rank], 10, world, torch.device("cpu"))
        out[rank] = (value, ms_max)
    finally:
        dist.destroy_process_group()


def test_job_rate_is_max_over_ranks_gloo():
    ms = [120.0, 250.0]
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank, args=(2, port, ms, out), nprocs=2, join=True)
        res = dict(out)
    for r in (0, 1):
        value, ms_max = res[r]
        assert ms_max == 250.0
        assert abs(value - 2 * 10 / 0.25) < 1e-9  # both ranks' steps over the slowest time


def test_reference_arm_silent_on_other_ranks():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
