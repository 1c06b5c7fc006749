"""The multi-rank plumbing of bench.py on the host cores: world-size-2 gloo ranks take the maximum of
their times and meet at the barriers; under torchrun the reference arm prints on rank 0 only."""
import json
import os
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as tdist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    bench.barrier(tdist)
    got = bench.max_over_ranks(tdist, 1.5 + rank)
    bench.barrier(tdist)
    tdist.destroy_process_group()
    q.put((rank, got))


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: 2.5, 1: 2.5}


def test_reference_arm_prints_on_rank_zero_only():
    # the ensemble's reference arm needs no oracle run: rank 0 prints its line, rank 1 nothing
    for rank, expect in ((0, True), (1, False)):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
        r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                            "ensemble"], env=env, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
        if expect:
            assert json.loads(lines[-1])["impl"] == "reference"
        else:
            assert lines == []


def test_reference_arm_other_ranks_do_no_work():
    """Rank 1 of the heated reference arm exits at once without output (rank 0 alone times the CPU
    arm)."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
