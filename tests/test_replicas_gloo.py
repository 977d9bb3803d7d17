"""Multi-GPU host logic (replicas only), run as world-size-2 gloo ranks on CPU.

Frames are independent, so N GPUs run N replicas: each rank takes its share
of the work, the timed region is bracketed by barriers, and the job time is
the maximum over ranks.  These tests run that plumbing (rav2d_b200/replicas.py,
used by bench.py) over gloo, including a rank that never joins.
"""
import os
import socket
import subprocess
import sys
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _env(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))


def _replica(rank, world, port, q):
    sys.path.insert(0, ROOT)
    _env(rank, world, port)
    from rav2d_b200 import replicas

    r, w = replicas.init("gloo", timeout_s=60)
    frames = [(640, 360), (1280, 720), (1920, 1080), (3840, 2160)] * 3
    mine = replicas.shard(frames, r, w)
    replicas.barrier()
    ms = 100.0 + 50.0 * r  # rank 1 is the slow one
    mx = replicas.max_over_ranks(ms)
    mpix = sum(a * b for a, b in mine) / 1e6
    units, ms_max, nrep = replicas.aggregate(mpix, ms)
    q.put((r, w, mine, mx, units / (ms_max / 1e3), nrep))
    replicas.finish()


def _lonely(rank, world, port, q):
    sys.path.insert(0, ROOT)
    _env(rank, world, port)
    from rav2d_b200 import replicas

    t0 = time.time()
    try:
        replicas.init("gloo", timeout_s=3)
        replicas.max_over_ranks(1.0)
        q.put(("joined", time.time() - t0))
    except Exception as e:  # the missing rank turns into an error, not a hang
        q.put((type(e).__name__, time.time() - t0))


def test_two_gloo_replicas_share_and_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_replica, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    (r0, w0, s0, mx0, v0, n0), (r1, w1, s1, mx1, v1, n1) = out
    assert (r0, r1, w0, w1) == (0, 1, 2, 2)
    assert mx0 == mx1 == 150.0  # max over ranks, seen by both
    assert sorted(s0 + s1) == sorted([(640, 360), (1280, 720), (1920, 1080), (3840, 2160)] * 3)
    assert len(s0) == len(s1) == 6
    # the job's rate: the units every rank processed over the slowest rank's
    # time, with the number of ranks that reported (the bench's n_gpus)
    assert n0 == n1 == 2
    mpix = sum(a * b for a, b in s0 + s1) / 1e6
    assert v0 == v1 == pytest.approx(mpix / 0.150)


def test_missing_rank_fails_fast():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_lonely, args=(0, 2, _free_port(), q))  # rank 1 never starts
    p.start()
    what, dt = q.get(timeout=120)
    p.join(60)
    assert what != "joined"
    assert dt < 60


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(_free_port()))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "3", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_bench_refuses_more_gpus_than_processes():
    """`bench.py --gpus 2` started as one process must fail, not print one
    process's rate as two GPUs' (the driver starts one process per GPU)."""
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--steps", "3", "--warmup", "3"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert r.stdout.strip() == ""
    assert "WORLD_SIZE is 1" in r.stderr
