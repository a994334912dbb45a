"""Host logic of the multi-rank (replica) bench path on CPU: world-size-2
gloo process group, max over ranks and the whole-job ERI throughput; the
reference arm on a non-zero rank exits without work."""
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = bench.max_over_ranks(100.0 + 50.0 * rank, dist, "cpu")
    eri = bench.eri_aggregate({"quartets": 1000, "ms": 10.0 + rank}, world, bench.max_over_ranks(10.0 + rank, dist, "cpu"))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ms, eri["ms"], eri["value"]))


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29611
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, eri_ms, eri_val in out:
        assert ms == 150.0            # the slowest rank's step time on every rank
        assert eri_ms == 11.0
        assert eri_val == pytest.approx(2 * 1000 / 11.0e-3)  # two replicas over the slowest time


def test_single_process_passthrough():
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


def test_reference_arm_nonzero_rank_exits_clean():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
