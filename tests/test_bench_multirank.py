"""World-size-2 check of bench.py's multi-rank bookkeeping on CPU (gloo): the
job time is the maximum over ranks and the whole-job value counts every rank's
bytes (band decomposition, weak scaling)."""
import os
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks([1.0 + rank, 10.0 - rank], dist, "cpu")
        out[rank] = (ms, bench.whole_job_gbs(1.0e9, world, ms[0]))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value():
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    for r in range(world):
        ms, gbs = out[r]
        assert ms == [2.0, 10.0]                       # maxima over the two ranks
        assert gbs == pytest.approx(2 * 1.0e9 / 2.0e-3 / 1e9)
