"""Partitioned solves on one GPU.

R ranks of an in-process group, each a context on its own CUDA stream driven by
its own host thread, exchange their ghost layers with stream-ordered device
copies.  Every owned patch must equal the one-rank solve bit for bit after
steps, ghost updates, regrids and repartitions, for every solver family, the
mixed form and the clawpack 5 update; the run loop takes the global CFL
maximum.  Failures are made on the host: a rank that never joins a collective,
and a rank whose call fails; the others get FCB_ERR_COMM within the time limit.
"""
import dataclasses
import threading
import time

import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu


def _ranks(R, fn, timeout_s=60.0):
    """fn(rank, comm, stream) on R threads; returns the results, raises the first error."""
    import forestclaw_b200 as fcb
    import torch

    comms = fcb.local_group(R, timeout_s=timeout_s)
    streams = [torch.cuda.Stream() for _ in range(R)]
    out, err = [None] * R, [None] * R

    def body(r):
        try:
            out[r] = fn(r, comms[r], streams[r].cuda_stream)
        except BaseException as e:  # noqa: BLE001 - re-raised below
            err[r] = e

    ts = [threading.Thread(target=body, args=(r,)) for r in range(R)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for e in err:
        if e is not None:
            raise e
    return out


def _owned(s, q_all):
    """Copies this rank's owned patches into the shared array; returns its range."""
    info = s.partition_info()
    s.get_q(q_all)
    return info["first"], info["count"]


def _check_partition(infos, n):
    first = 0
    for r, (f, c) in enumerate(infos):
        assert f == first, (r, infos)
        first += c
    assert first == n


def _stepped(opts, R, steps, dt, regrid=False):
    """(serial q, partitioned q, serial leaves, partitioned leaves per rank, cfls) after `steps` macro steps."""
    import forestclaw_b200 as fcb

    s = fcb.Solver(opts)
    s.initialize()
    serial_cfl = []
    t = 0.0
    for _ in range(steps):
        serial_cfl.append(s.advance_all_levels(t, dt))
        t += dt
        if regrid:
            s.regrid()
    q_ref = s.get_q()
    leaves_ref = s.leaves()
    n = s.num_patches
    q_all = np.full_like(q_ref, np.nan)

    def rank(r, comm, stream):
        d = fcb.Solver(opts, stream=stream, comm=comm)
        d.initialize()
        cfl = []
        tt = 0.0
        for _ in range(steps):
            cfl.append(d.global_maximum(d.advance_all_levels(tt, dt)))
            tt += dt
            if regrid:
                d.regrid()
        rng = _owned(d, q_all)
        return d.leaves(), rng, cfl, d.counters()

    res = _ranks(R, rank)
    for leaves, _, cfl, _ in res:
        assert leaves == leaves_ref
        assert cfl == serial_cfl
    _check_partition([r[1] for r in res], n)
    return q_ref, q_all, res


@pytest.mark.parametrize("R", [2, 3])
def test_uniform_swirl_bit_exact(gpu_lib, R):
    cfg = cases.swirl_uniform(level=4)
    q_ref, q_all, res = _stepped(cases.to_options(cfg), R, steps=12, dt=0.9 / 256)
    assert np.array_equal(q_all, q_ref)
    # every rank updated its own patches only
    assert sum(r[3]["count_single_step"] for r in res) == 12 * 256


def test_amr_shallow_water_regrid_bit_exact(gpu_lib):
    cfg = cases.radialdam_amr(seed=2, minlevel=2, maxlevel=4, mx=16)
    q_ref, q_all, _ = _stepped(cases.to_options(cfg), 3, steps=6, dt=0.9 / (16 * 16) / 1.5, regrid=True)
    assert np.array_equal(q_all, q_ref)


def test_amr_euler_run_loop_bit_exact(gpu_lib):
    """fcb_run: adaptive dt from the global CFL maximum, regrid every step, repartition."""
    import forestclaw_b200 as fcb

    cfg = cases.quadrants_amr(seed=1, minlevel=2, maxlevel=5, mx=8, tfinal=0.05)
    opts = cases.to_options(cfg)
    s = fcb.Solver(opts)
    s.initialize()
    s.run()
    q_ref = s.get_q()
    q_all = np.full_like(q_ref, np.nan)
    c_ref = s.counters()

    def rank(r, comm, stream):
        d = fcb.Solver(opts, stream=stream, comm=comm)
        d.initialize()
        d.run()
        _owned(d, q_all)
        return d.counters(), d.leaves(), d.conservation_check()

    res = _ranks(4, rank)
    for c, leaves, mass in res:
        assert c["count_amr_advance"] == c_ref["count_amr_advance"]
        assert c["count_amr_new_domain"] == c_ref["count_amr_new_domain"]
        assert leaves == s.leaves()
        assert np.array_equal(mass, s.conservation_check())
    assert np.array_equal(q_all, q_ref)


def test_weighted_partition_balances_subcycled_work(gpu_lib):
    import forestclaw_b200 as fcb

    cfg = cases.radialdam_amr(seed=0, minlevel=2, maxlevel=5, mx=8)
    opts = cases.to_options(cfg)

    def rank(r, comm, stream):
        d = fcb.Solver(opts, stream=stream, comm=comm)
        d.initialize()
        info = d.partition_info()
        lv = [d.patch_info(p)[0] for p in range(info["first"], info["first"] + info["count"])]
        return info, lv, d.leaves()

    res = _ranks(3, rank)
    _check_partition([(i["first"], i["count"]) for i, _, _ in res], len(res[0][2]))
    w = [sum(2 ** l for l in lv) for _, lv, _ in res]
    total = sum(w)
    leaves = res[0][2]
    maxw = max(2 ** l for l, _, _ in leaves)
    # each range holds about a third of the weight (a family moves a cut by at most 4 leaves)
    for wr in w:
        assert abs(wr - total / 3) <= 4 * maxw
    # no cut splits a complete family of leaves
    for i, _, _ in res[1:]:
        c = i["first"]
        for a in range(max(0, c - 3), c):
            fam = leaves[a:a + 4]
            if len(fam) == 4 and len({l for l, _, _ in fam}) == 1:
                lvl, x, y = fam[0]
                h = 1 << (28 - lvl)
                sib = [(lvl, x + (k & 1) * h, y + (k >> 1) * h) for k in range(4)]
                if x % (2 * h) == 0 and y % (2 * h) == 0 and list(fam) == sib:
                    assert not (a < c < a + 4)


def test_bathymetry_mixed_precision_bit_exact(gpu_lib):
    import forestclaw_b200 as fcb

    cfg = cases.bathy_lake(level=3, mx=16, seed=3, minlevel=2, maxlevel=4)
    opts = cases.to_options(cfg)
    opts.precision = fcb.PRECISION_MIXED
    q_ref, q_all, _ = _stepped(opts, 2, steps=4, dt=0.002, regrid=True)
    assert np.array_equal(q_all, q_ref)


def test_clawpack5_update_bit_exact(gpu_lib):
    cfg = dataclasses.replace(cases.swirl_uniform(level=3), claw_version=5)
    opts = cases.to_options(cfg)
    q_ref, q_all, _ = _stepped(opts, 2, steps=5, dt=0.9 / 128)
    assert np.array_equal(q_all, q_ref)


def test_more_ranks_than_work(gpu_lib):
    """Ranks that own few or no leaves still take part in every collective."""
    cfg = cases.swirl_uniform(level=1)
    q_ref, q_all, res = _stepped(cases.to_options(cfg), 6, steps=3, dt=0.9 / 32)
    assert np.array_equal(q_all, q_ref)
    assert min(r[1][1] for r in res) == 0


def test_rank_that_never_joins_times_out(gpu_lib):
    import forestclaw_b200 as fcb

    opts = cases.to_options(cases.swirl_uniform(level=2))

    def rank(r, comm, stream):
        d = fcb.Solver(opts, stream=stream, comm=comm)
        d.initialize()
        if r == 1:
            return None  # leaves between steps, without joining the ghost update
        t0 = time.monotonic()
        with pytest.raises(fcb.FcbError) as e:
            d.ghost_update(2, 2)
        return e.value.code, time.monotonic() - t0

    res = _ranks(2, rank, timeout_s=2.0)
    code, waited = res[0]
    assert code == 6  # FCB_ERR_COMM
    assert 1.5 < waited < 30.0


def test_failed_rank_stops_the_others(gpu_lib):
    import forestclaw_b200 as fcb

    opts = cases.to_options(cases.swirl_uniform(level=2))
    go = threading.Event()

    def rank(r, comm, stream):
        d = fcb.Solver(opts, stream=stream, comm=comm)
        if r == 1:
            with pytest.raises(fcb.FcbError) as e:  # fails on this rank: not initialised
                d.advance_all_levels(0.0, 0.01)
            go.set()
            return e.value.code, 0.0
        d.initialize()
        go.wait(30)
        t0 = time.monotonic()
        with pytest.raises(fcb.FcbError) as e:
            d.ghost_update(2, 2)
        return e.value.code, time.monotonic() - t0

    res = _ranks(2, rank, timeout_s=60.0)
    assert res[1][0] == 3  # FCB_ERR_STATE on the failing rank
    assert res[0][0] == 6 and res[0][1] < 10.0  # the other learns at once, not after 60 s


def test_partitioned_option_checks(gpu_lib):
    import forestclaw_b200 as fcb

    comms = fcb.local_group(2)
    opts = cases.to_options(dataclasses.replace(O.radialdam_regression(), minlevel=2, maxlevel=3))
    opts.time_sync = 1
    with pytest.raises(fcb.FcbError) as e:
        fcb.Solver(opts, comm=comms[0])
    assert e.value.code == 1


def test_nccl_communicator_one_rank(gpu_lib):
    """The NCCL communicator (loaded at run time, non-blocking, bounded waits)
    as a one-rank partitioned solve: initialisation, the global maximum, the
    gathered tags and the rank's own exchange path; equal to the plain solve."""
    import forestclaw_b200 as fcb

    comm = fcb.nccl_comm(fcb.nccl_unique_id(), 0, 1, timeout_s=60.0)
    opts = cases.to_options(cases.radialdam_amr(seed=1, minlevel=2, maxlevel=4, mx=16))
    s = fcb.Solver(opts)
    d = fcb.Solver(opts, comm=comm)
    s.initialize()
    d.initialize()
    t, dt = 0.0, 0.002
    for _ in range(4):
        assert d.global_maximum(d.advance_all_levels(t, dt)) == s.advance_all_levels(t, dt)
        t += dt
        assert d.regrid() == s.regrid()
    assert d.leaves() == s.leaves()
    assert np.array_equal(d.get_q(), s.get_q())
    assert np.array_equal(d.conservation_check(), s.conservation_check())
    assert d.partition_info() == {"rank": 0, "nranks": 1, "first": 0, "count": s.num_patches}


@pytest.mark.parametrize("subcycle,weighted", [(0, 1), (1, 0)])
def test_partitioned_schedule_variants(gpu_lib, subcycle, weighted):
    """Non-subcycled steps (every level with the fine dt, ghost fills over all
    levels) and an unweighted partition, on a mesh of several levels."""
    cfg = dataclasses.replace(cases.quadrants_amr(seed=1, minlevel=2, maxlevel=5, mx=8), subcycle=subcycle)
    opts = cases.to_options(cfg)
    opts.weighted_partition = weighted
    q_ref, q_all, _ = _stepped(opts, 3, steps=3, dt=0.9 / (8 * 32) / 1.5 / (1 if subcycle else 8), regrid=True)
    assert np.array_equal(q_all, q_ref)


def test_partitioned_ascii_frame(gpu_lib, tmp_path):
    """fcb_output_ascii of a 3-rank solve: the header from rank 0, then the
    ranks' patches in rank order; equal to the one-rank frame apart from the
    mpi_rank line of each grid header."""
    import forestclaw_b200 as fcb

    cfg = cases.radialdam_amr(seed=1, minlevel=2, maxlevel=4, mx=8)
    opts = cases.to_options(cfg)
    dt = 0.002
    s = fcb.Solver(opts)
    s.initialize()
    s.advance_all_levels(0.0, dt)
    (tmp_path / "one").mkdir()
    (tmp_path / "three").mkdir()
    s.output_ascii(7, str(tmp_path / "one"))

    def rank(r, comm, stream):
        d = fcb.Solver(opts, stream=stream, comm=comm)
        d.initialize()
        d.global_maximum(d.advance_all_levels(0.0, dt))
        d.output_ascii(7, str(tmp_path / "three"))
        return d.partition_info()

    infos = _ranks(3, rank)
    assert (tmp_path / "one" / "fort.t0007").read_text() == (tmp_path / "three" / "fort.t0007").read_text()
    one = (tmp_path / "one" / "fort.q0007").read_text().split("\n")
    three = (tmp_path / "three" / "fort.q0007").read_text().split("\n")
    assert len(one) == len(three)
    owner = {}
    for i in infos:
        for p in range(i["first"], i["first"] + i["count"]):
            owner[p] = i["rank"]
    grid = None
    for a, b in zip(one, three):
        if a.endswith("grid_number"):
            grid = int(a.split()[0])
        if a.endswith("mpi_rank"):
            assert int(b.split()[0]) == owner[grid]
        else:
            assert a == b
    assert len(set(owner.values())) == 3


def test_partitioned_state_io_and_patch_protocol(gpu_lib):
    """set_q / get_q move only the owned patches at their places in the
    all-leaves layout; the per-patch protocol (single_step_update) accepts a
    rank's own patches and rejects the others'."""
    import forestclaw_b200 as fcb

    opts = cases.to_options(cases.swirl_uniform(level=3))
    s = fcb.Solver(opts)
    s.initialize()
    q0 = s.get_q()
    rng = np.random.default_rng(5)
    q1 = q0 + rng.uniform(0.0, 1e-3, size=q0.shape)
    out = np.full_like(q0, np.nan)

    def rank(r, comm, stream):
        d = fcb.Solver(opts, stream=stream, comm=comm)
        d.initialize()
        info = d.partition_info()
        f, c = info["first"], info["count"]
        d.set_q(q1)
        d.get_q(out)
        mine, other = f, (f + c) % d.num_patches
        cfl = d.single_step_update(mine, 0.0, 0.001, 0, 1)
        with pytest.raises(fcb.FcbError) as e:
            d.single_step_update(other, 0.0, 0.001, 0, 1)
        return cfl, e.value.code

    res = _ranks(2, rank)
    assert np.array_equal(out, q1)
    for cfl, code in res:
        assert cfl > 0.0 and code == 1
