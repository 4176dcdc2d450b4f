"""bench.py under torchrun: every rank times its own replica and the job's
rate divides all ranks' units by the slowest rank's time (an all-reduce MAX
every rank takes).  Run here as two gloo ranks on the CPU; the reference
arm's non-zero ranks exit without work."""
from __future__ import annotations

import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rate, ms_max = bench.job_rate(dist, [10.0, 20.0][rank], 5, world, device="cpu")
        q.put((rank, rate, ms_max))
    finally:
        dist.destroy_process_group()


def test_job_rate_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for _, rate, ms_max in got:
        assert ms_max == 20.0 and abs(rate - 2 * 5 / 0.020) < 1e-9


def test_reference_arm_other_ranks_exit():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], capture_output=True, text=True, timeout=120, env=env, cwd=ROOT)
    assert r.returncode == 0 and r.stdout.strip() == ""
