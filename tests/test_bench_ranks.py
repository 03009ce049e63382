"""Multi-rank logic of bench.py on the CPU (gloo, two ranks): the job's time is its slowest rank's,
the whole-job rate counts every rank's paths, replicas render distinct seeded scenes, and the
reference arm runs on rank 0 only (the other ranks exit 0 without output)."""
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


def _rank(rank, world, port, times, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        slowest = bench.max_over_ranks(times[rank], dist, "cpu")
        rate = bench.whole_job_rate(1_000_000, world, slowest / 1e3)
        q.put((rank, slowest, rate))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_count_every_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    times = [120.0, 180.0]
    procs = [ctx.Process(target=_rank, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, rate in got:
        assert slowest == 180.0
        assert rate == pytest.approx(2 * 1_000_000 / 0.18)


def test_one_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(42.5) == 42.5
    assert bench.whole_job_rate(10, 1, 2.0) == 5.0


def test_replicas_render_distinct_seeded_scenes():
    from jarabotransientrendering_b200 import scenes as S
    import numpy as np
    a, b = S.WORKLOADS["icosphere"](seed=1), S.WORKLOADS["icosphere"](seed=2)
    assert a.seed != b.seed
    assert a.paths_per_frame() == b.paths_per_frame()            # same work per rank (weak scaling)
    va, _, _ = a.flatten()
    vb, _, _ = b.flatten()
    assert va.shape == vb.shape and not np.array_equal(va, vb)


def test_reference_arm_prints_nothing_on_other_ranks():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                         capture_output=True, text=True, env=env, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == ""
