"""The N > 1 partitioned path on CPU: the library's host-only planning query
(fcb_partition_plan, no device call) on two gloo ranks.  Each rank plans its
own part of the same meshes (uniform, and AMR meshes the oracle builds with
regrids), the ranks gather their plans over gloo, and every exchange must be
matched: what rank a sends to rank b is what b expects from a, in both ghost
update exchanges, for full and time-interpolated updates.  The owned ranges
tile the leaves, and a one-rank plan exchanges nothing."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _meshes():
    """(options, leaves, ghost updates) for a uniform mesh and three AMR meshes."""
    import cases
    import oracle as O

    out = []
    u = cases.swirl_uniform(level=3)
    s = O.OracleSolver(u)
    s.initialize()
    out.append((cases.to_options(u), s.leaves(), [(3, 3, 0)]))
    for cfg, steps in ((cases.radialdam_amr(seed=0, minlevel=2, maxlevel=5, mx=16), 0),
                       (cases.radialdam_amr(seed=3, minlevel=2, maxlevel=5, mx=16), 3),
                       (cases.quadrants_amr(seed=0, minlevel=2, maxlevel=5, mx=8), 2)):
        s = O.OracleSolver(cfg)
        s.initialize()
        t, dt = 0.0, 0.002
        for _ in range(steps):
            s.advance(t, dt)
            t += dt
            s.regrid()
        lv = [l for l, _, _ in s.leaves()]
        lo, hi = min(lv), max(lv)
        updates = [(lo, hi, 0)] + [(l, hi, 1) for l in range(lo + 1, hi + 1)]
        out.append((cases.to_options(cfg), s.leaves(), updates))
    return out


def _check_matched(plans, n):
    R = len(plans)
    first = 0
    for r in range(R):
        assert plans[r]["first"] == first
        first += plans[r]["count"]
    assert first == n
    for a in range(R):
        for b in range(R):
            for x in ("x1", "x2"):
                assert plans[a][x + "_send"][b] == plans[b][x + "_recv"][a], (a, b, x)
        assert plans[a]["x1_send"][a] == 0 and plans[a]["x2_send"][a] == 0


def _rank_main(rank, world, port, out):
    import datetime
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "tests")]
    import forestclaw_b200 as fcb

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        checked = 0
        for opts, leaves, updates in _meshes():
            for mn, mxl, ti in updates:
                mine = fcb.partition_plan(opts, leaves, rank, world, mn, mxl, ti)
                plans = [None] * world
                dist.all_gather_object(plans, mine)
                _check_matched(plans, len(leaves))
                checked += 1
        out[rank] = checked
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_plan_matched_exchanges():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert set(res) == {0, 1}
    assert res[0] == res[1] and res[0] >= 7


@pytest.mark.parametrize("R", [1, 3, 5])
def test_plans_matched_for_more_ranks(R):
    import forestclaw_b200 as fcb

    for opts, leaves, updates in _meshes():
        for mn, mxl, ti in updates:
            plans = [fcb.partition_plan(opts, leaves, r, R, mn, mxl, ti) for r in range(R)]
            _check_matched(plans, len(leaves))
            if R == 1:
                assert plans[0]["ghosts"] == 0
                assert sum(plans[0]["x1_recv"]) == 0 and sum(plans[0]["x2_recv"]) == 0


def test_interpolation_sources_cross_ranks_in_the_second_exchange():
    """On an AMR mesh cut across a coarse/fine boundary some rank receives coarse
    patches in the second exchange, and only coarse/fine meshes need it."""
    import forestclaw_b200 as fcb

    meshes = _meshes()
    opts, leaves, updates = meshes[0]
    assert all(sum(fcb.partition_plan(opts, leaves, r, 3, 3, 3)["x2_recv"]) == 0 for r in range(3))
    opts, leaves, updates = meshes[2]
    mn, mxl, _ = updates[0]
    assert sum(sum(fcb.partition_plan(opts, leaves, r, 3, mn, mxl, 0)["x2_recv"]) for r in range(3)) > 0


def test_invalid_leaves_rejected():
    import forestclaw_b200 as fcb

    import cases

    opts = cases.to_options(cases.swirl_uniform(level=1))
    h = 1 << 27
    good = [(1, 0, 0), (1, h, 0), (1, 0, h), (1, h, h)]
    assert fcb.partition_plan(opts, good, 0, 2, 1, 1)["count"] + fcb.partition_plan(opts, good, 1, 2, 1, 1)["count"] == 4
    for bad in ([(1, h, 0), (1, 0, 0), (1, 0, h), (1, h, h)],  # not in Morton order
                [(1, 0, 0), (1, h, 0), (1, 0, h)],  # a hole
                [(1, 0, 0), (1, h + 1, 0), (1, 0, h), (1, h, h)]):  # off the level's grid
        with pytest.raises(fcb.FcbError) as e:
            fcb.partition_plan(opts, bad, 0, 2, 1, 1)
        assert e.value.code == 1
    with pytest.raises(fcb.FcbError):
        fcb.partition_plan(opts, good, 2, 2, 1, 1)
