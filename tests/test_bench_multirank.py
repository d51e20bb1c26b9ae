"""CPU tests of bench.py's multi-rank plumbing (gloo, world_size 2): the
timing reduction is the max over ranks, the whole-job value counts every
rank's steps, and the reference arm does no work on ranks other than 0."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    from datetime import timedelta

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    total_ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
    m = bench._max_over_ranks(dist, total_ms)
    q.put((rank, m, bench._job_gflops(2e12, world, 10, m)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_job_value_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, value in out:
        assert m == 150.0  # every rank sees the slowest rank's time
        # 2 ranks x 10 steps x 2 TFLOP over 150 ms
        assert value == pytest.approx(2e12 * 2 * 10 / 0.150 * 1e-9)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2"], capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
