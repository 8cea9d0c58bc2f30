"""The N > 1 path on CPU: two gloo ranks, each advancing an independent
replica (the oracle stands in for the GPU solve), with the benchmark's
reductions of the measurement (slowest rank's time, total cell updates)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import datetime
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "tests")]
    import cases
    import oracle as O
    from forestclaw_b200 import replicas

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg = cases.radialdam_amr(seed=replicas.replica_seed(0, rank), minlevel=1, maxlevel=2, mx=8, tfinal=0.02)
        s = O.OracleSolver(cfg)
        s.initialize()
        dist.barrier()
        for k in range(3):
            s.advance(k * 0.004, 0.004)
        cells = s.counters()["count_single_step"] * cfg.mx * cfg.my
        ms_local = 10.0 + rank  # a stand-in for the rank's device time
        ms_max, total = replicas.aggregate(ms_local, cells, dist)
        out[rank] = (ms_max, total, cells, s.all_q().sum(), cfg.pparams[2])
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas_reduce_time_and_cells():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert set(res) == {0, 1}
    for r in range(world):
        ms_max, total, _, _, _ = res[r]
        assert ms_max == 11.0  # the slowest rank's time on every rank
        assert total == res[0][2] + res[1][2]
    # independent replicas: different seeded data, different results
    assert res[0][4] != res[1][4]
    assert res[0][3] != res[1][3]


def test_aggregate_single_process():
    from forestclaw_b200 import replicas

    assert replicas.aggregate(1.5, 7, None) == (1.5, 7)
