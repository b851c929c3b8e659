"""The multi-rank arithmetic of bench.py on CPU (gloo, world size 2): every
rank takes part in the max-reduction of the timed region, and the reported
value is the work of all replicas over the slowest rank's time.  The path has
no data-path collective (independent replicas), so this is its only
cross-rank step."""
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(1.0 + 2.0 * rank, world, "cpu")   # rank 1 is the slow one
        v = bench.aggregate_rate(10.0, 4, world, t)
        q.put((rank, t, v))
    finally:
        dist.destroy_process_group()


def test_two_ranks_report_the_slowest_time_and_all_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    assert all(p.exitcode == 0 for p in ps)
    out = sorted(q.get(timeout=5) for _ in range(2))
    for rank, t, v in out:
        assert t == pytest.approx(3.0)
        assert v == pytest.approx(10.0 * 4 * 2 / 3.0)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(2.5, 1, "cpu") == 2.5
    assert bench.aggregate_rate(6.0, 2, 1, 3.0) == pytest.approx(4.0)
