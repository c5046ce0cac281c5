"""The multi-GPU path of bench.py is replicas only: each rank solves its own realisation
(seed + rank) and the only collective is the max over ranks of the timed duration.  Checked
here with two gloo ranks on the CPU (no GPU needed)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
    got = bench.max_over_ranks(dist, ms, "cpu")
    q.put((rank, got, bench.replica_seed(1000, rank), bench.replicas_value(world, 5, got)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time_and_distinct_seeds():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert [o[1] for o in out] == [150.0, 150.0]  # both ranks see the slowest rank's time
    assert out[0][2] != out[1][2]                 # independent realisations
    assert out[0][3] == pytest.approx(2 * 5 / 0.150)  # whole-job solves/s
