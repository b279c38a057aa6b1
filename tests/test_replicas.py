"""The multi-GPU path on the host, without a GPU: replicas over a world_size-2
gloo process group agree on the slowest rank's times, the whole-job rate
counts every rank's work, and the non-zero ranks of the reference arm exit
without work or output."""
import datetime
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


def _worker(rank, world, port, q):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from highmap_b200.replicas import job_rate, max_over_ranks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r's step took 100 + r ms; its two parts differ in which rank is slower
        times = max_over_ranks([100.0 + rank, 40.0 + 10.0 * (world - 1 - rank), 60.0 + rank], dist, "cpu")
        dist.barrier()
        q.put((rank, times, job_rate(world, 5, 1000.0, times[0])))
    finally:
        dist.destroy_process_group()


def test_replicas_over_gloo():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = {}
    try:
        for _ in procs:
            rank, times, rate = q.get(timeout=120)
            results[rank] = (times, rate)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert sorted(results) == [0, 1]
    for times, rate in results.values():
        assert times == [101.0, 50.0, 61.0]
        assert rate == pytest.approx(2 * 5 * 1000.0 / 0.101)
    assert all(p.exitcode == 0 for p in procs)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    from highmap_b200.replicas import job_rate, max_over_ranks
    assert max_over_ranks([3.0, 1.5]) == [3.0, 1.5]
    assert job_rate(1, 2, 10.0, 1000.0) == pytest.approx(20.0)
    with pytest.raises(ValueError):
        job_rate(1, 1, 1.0, 0.0)


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


@pytest.mark.parametrize("form", ["tblock", "sweep"])
def test_single_gpu_forms_other_ranks_exit_quietly(form):
    """The forms that measure one GPU run on rank 0 of a torchrun launch;
    the other ranks exit 0 before any device call."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--form", form, "--sizes", "128"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
