"""Multi-rank plumbing of bench.py on CPU: world_size-2 gloo ranks (no GPU).

The field-construction path does not shard: each rank builds its own realisation and the
only collective is the timing reduction, the maximum of the per-rank device times.  These
tests run that reduction on gloo ranks and check the whole-job rate, and that the reference
arm does its work on rank 0 alone.
"""
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
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
        t = bench.max_over_ranks(ms, dist, "cpu")
        rate = bench.whole_job_rate(world, 3, 64, t)
        dist.barrier()
        q.put((rank, t, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, t, rate in got:
        assert t == 150.0                                   # every rank sees the slowest time
        assert rate == pytest.approx(2 * 3 * 64 ** 3 / 0.150 / 1e6)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5) == 12.5
    assert bench.whole_job_rate(1, 2, 256, 1000.0) == pytest.approx(2 * 256 ** 3 / 1e6)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_reference_arm_estimate_tracks_a_whole_oracle_run(orc):
    """The reference arm times a bounded sample (the first tube of every level on a reduced grid,
    the spectral path and statistics on at most 256^3) and scales it to a whole field.  On cfg0,
    small enough to run whole, the estimate lands within a factor 2 of the measured whole run."""
    import time

    sys.path.insert(0, ROOT)
    import bench
    from fastweavturb_b200.configs import cfg0
    from helpers import oracle_inputs

    w = cfg0(seed=0)
    est, parts = bench.cpu_sample_estimate(w)
    p, cl = oracle_inputs(orc, w)
    t = time.perf_counter()
    orc.run(p, cl)
    whole = time.perf_counter() - t
    assert 0.5 * whole <= est <= 2.0 * whole, (est, whole)
    assert "grids [64, 64, 64]" in parts["sample"]
