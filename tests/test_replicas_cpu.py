"""The multi-GPU form of bench.py runs one independent index per rank
(replicas, weak scaling); its only exchange is the maximum of the per-rank
times.  This runs that reduction and the whole-job rate on two gloo ranks on
the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # Rank r's timed region took (10 + r) ms for the device-resident steps
        # and (20 - r) ms end to end.
        total_ms, e2e_ms = bench.max_over_ranks(dist, [10.0 + rank, 20.0 - rank], "cpu")
        out[rank] = (total_ms, e2e_ms, bench.whole_job_rate(1 << 20, world, total_ms))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_take_the_slowest_rank():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        total_ms, e2e_ms, rate = res[r]
        assert total_ms == 11.0 and e2e_ms == 20.0
        # Both ranks' requests over the slower rank's 11 ms.
        assert abs(rate - 2 * (1 << 20) / 0.011 / 1e6) < 1e-6
