"""The multi-rank path of bench.py on CPU: two gloo ranks (replicas, one
GPU each on a B200 node), barrier and max over ranks, whole-job rate, and the
reference arm's non-zero ranks exiting without work."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    ranks = bench.RankGroup.init("gloo", world, timeout_s=60)
    ranks.barrier()
    m = ranks.max(1.5 + rank)             # per-rank time: the slowest rank sets the job time
    rate = bench.whole_job_rate(16, world, m)
    ranks.barrier()
    ranks.pg.destroy_process_group()
    out.put((rank, m, rate))


def test_two_gloo_ranks_take_the_max():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [2.5, 2.5]
    assert all(abs(g[2] - 16 * 2 / 2.5) < 1e-9 for g in got)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    r = bench.RankGroup.init("gloo", 1)
    r.barrier()
    assert r.max(3.0) == 3.0 and r.pg is None


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0
    assert p.stdout.strip() == ""
