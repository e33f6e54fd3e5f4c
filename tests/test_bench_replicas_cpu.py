"""The N > 1 path of bench.py on CPU: world_size-2 `gloo` ranks.

The path does not shard (independent replicas), so the multi-rank logic is the
max-over-ranks time, the whole-job value, and the reference arm running on
rank 0 only.  These run as two spawned processes over gloo on 127.0.0.1."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

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
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = [1.5, 2.25][rank]
        mx = bench.max_over_ranks(ms, dist, "cpu")
        e = bench.max_over_ranks([0.7, 0.4][rank], dist, "cpu")
        dist.barrier()
        q.put((rank, mx, e, bench.whole_job_gbs(world, 10**9, mx)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, mx, e, gbs in res:
        assert mx == 2.25 and e == 0.7
        assert gbs == pytest.approx(2 * 1e9 / 2.25e-3 / 1e9)


def test_reference_arm_nonzero_rank_exits_without_work(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")

    class A:
        rows, steps, warmup = 16, 1, 0
    assert bench.run_reference(A()) == 0


def test_single_rank_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0
    assert bench.whole_job_gbs(1, 2 * 10**9, 1.0) == pytest.approx(2000.0)
