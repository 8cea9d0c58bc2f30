"""Ensemble serving: continuous batching of independent solves.

A served solve must give the same result alone and in a mix of concurrent
solves (batching only changes which launch a patch is in), and the same
result as fcb_run on the same options, subcycled or not.  Both are checked bit
for bit, in FP64 and in the mixed FP32/FP64 form; a subcycled served solve is
also checked against the oracle's fclaw2d_run.
"""
import dataclasses

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def _dam_cfg(seed, maxlevel, mx=16, tfinal=0.03, subcycle=0):
    return cases.replace(cases.radialdam_amr(seed=seed, minlevel=2, maxlevel=maxlevel, mx=mx, tfinal=tfinal),
                         subcycle=subcycle)


def _dam(seed, maxlevel, mx=16, tfinal=0.03, precision=0, subcycle=0):
    o = cases.to_options(_dam_cfg(seed, maxlevel, mx, tfinal, subcycle))
    o.precision = precision
    return o


def _serve(reqs, budget=1 << 40, stagger_rounds=0):
    """Submit requests (staggered by `stagger_rounds` rounds), run to idle,
    return the final states in submission order."""
    from forestclaw_b200.serve import DONE, Server

    sv = Server(budget)
    ids, out = [], {}
    pending = list(reqs)
    while pending or any(sv.status(i).state < DONE for i in ids):
        if pending:
            ids.append(sv.submit(pending.pop(0)))
            for _ in range(stagger_rounds):
                sv.round()
        else:
            sv.round()
    for k, i in enumerate(ids):
        st = sv.status(i)
        assert st.state == DONE, sv.error(i)
        out[k] = sv.get_q(i)
        sv.release(i)
    sv.close()
    return [out[k] for k in range(len(reqs))]


@pytest.mark.parametrize("subcycle", [0, 1])
def test_served_solve_equals_run(gpu_lib, subcycle):
    import forestclaw_b200 as fcb

    o = _dam(seed=0, maxlevel=4, subcycle=subcycle)
    d = fcb.Solver(dataclasses.replace(o))
    d.initialize()
    d.run()
    (q_served,) = _serve([o])
    assert np.array_equal(q_served, d.get_q())


def test_subcycled_served_solve_equals_oracle(gpu_lib):
    """fclaw2d_run of the oracle (subcycled levels 2-5, time interpolation,
    adaptive dt, regrid every macro step) against the served solve, every
    patch array bit for bit."""
    import oracle as O

    cfg = _dam_cfg(seed=3, maxlevel=5, mx=16, tfinal=0.02, subcycle=1)
    o = O.OracleSolver(cfg)
    o.initialize()
    o.run()
    (q_served,) = _serve([cases.to_options(cfg)])
    assert q_served.shape == o.all_q().shape
    assert np.array_equal(q_served, o.all_q())


@pytest.mark.parametrize("precision,subcycle", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_alone_and_in_the_mix_are_identical(gpu_lib, precision, subcycle):
    reqs = [_dam(seed=s, maxlevel=ml, tfinal=tf, precision=precision, subcycle=subcycle)
            for s, ml, tf in [(1, 3, 0.03), (2, 5, 0.02), (3, 4, 0.04), (4, 3, 0.01)]]
    alone = [_serve([r])[0] for r in reqs]
    mixed = _serve(reqs, stagger_rounds=3)
    for k, (a, m) in enumerate(zip(alone, mixed)):
        assert np.array_equal(a, m), f"request {k}"


def test_two_patch_shapes_and_a_memory_budget(gpu_lib):
    """Requests with mx 16 and 32 go to separate launches of the same round; a
    budget that holds about one solve serialises admission but every request
    completes with the same result as alone."""
    from forestclaw_b200.serve import DONE, Server

    reqs = [_dam(seed=5, maxlevel=3, mx=16), _dam(seed=6, maxlevel=3, mx=32), _dam(seed=7, maxlevel=3, mx=16)]
    alone = [_serve([r])[0] for r in reqs]
    sv = Server(1 << 40)
    ids = [sv.submit(r) for r in reqs]
    sv.round()
    _, rounds0, launches0 = sv.clock()
    sv.round()
    _, rounds1, launches1 = sv.clock()
    assert launches1 - launches0 == 2  # one launch per patch shape
    sv.run_until_idle()
    for k, i in enumerate(ids):
        assert sv.status(i).state == DONE
        assert np.array_equal(sv.get_q(i), alone[k])
    sv.close()
    # tiny budget: at most one solve on the device at a time
    sv = Server(1)
    ids = [sv.submit(r) for r in reqs]
    spans = []
    sv.run_until_idle()
    for k, i in enumerate(ids):
        st = sv.status(i)
        assert st.state == DONE
        spans.append((st.start_s, st.finish_s))
        assert np.array_equal(sv.get_q(i), alone[k])
    spans.sort()
    for (s0, f0), (s1, f1) in zip(spans, spans[1:]):
        assert s1 >= f0 - 1e-9  # admitted only after the previous one finished
    sv.close()


def test_poisson_stream_reports_latencies(gpu_lib):
    from forestclaw_b200.serve import Server, poisson_stream

    reqs = [_dam(seed=10 + k, maxlevel=3 + (k % 2), tfinal=0.01) for k in range(6)]
    sv = Server(1 << 40)
    res = poisson_stream(sv, reqs, rate=200.0, seed=1)
    sv.close()
    assert len(res.latencies) == 6 and res.failed == 0
    assert res.pct(99) >= res.pct(50) > 0
    assert res.cell_updates > 0 and res.launches >= res.rounds


def test_work_limit_serialises_admission(gpu_lib):
    """A work limit smaller than any solve's cells admits one solve at a time
    (each starts after the previous one finished); the results equal the
    solves run alone."""
    from forestclaw_b200.serve import DONE, Server

    reqs = [_dam(seed=20 + k, maxlevel=3 + (k % 2), subcycle=1) for k in range(3)]
    alone = [_serve([r])[0] for r in reqs]
    sv = Server(1 << 40)
    sv.set_work_limit(1)
    ids = [sv.submit(r) for r in reqs]
    sv.run_until_idle()
    spans = []
    for k, i in enumerate(ids):
        st = sv.status(i)
        assert st.state == DONE
        spans.append((st.start_s, st.finish_s))
        assert np.array_equal(sv.get_q(i), alone[k])
    spans.sort()
    for (s0, f0), (s1, f1) in zip(spans, spans[1:]):
        assert s1 >= f0 - 1e-9
    sv.close()


def _retry_cfg(scale):
    base = cases.radialdam_amr(seed=0, minlevel=2, maxlevel=4, mx=16, tfinal=0.05)
    return cases.replace(base, initial_dt=scale * base.initial_dt)


def test_served_cfl_retry_equals_run(gpu_lib):
    """A served subcycled solve whose first macro step exceeds max_cfl (initial
    dt 1.5 times too large): the saved state is restored and the step retaken
    with the smaller dt, as fcb_run does; the result is bit for bit fcb_run's."""
    import forestclaw_b200 as fcb

    o = cases.to_options(_retry_cfg(1.5))
    d = fcb.Solver(dataclasses.replace(o))
    d.initialize()
    d.run()
    c = d.counters()
    assert c["count_amr_advance"] > c["count_amr_regrid"]  # a step was retaken
    (q_served,) = _serve([o])
    assert np.array_equal(q_served, d.get_q())


def test_failed_solve_leaves_the_mix_intact(gpu_lib):
    """A solve with a negative depth outside the dam (every speed there a NaN,
    so its CFL maximum is a NaN) fails with FCB_ERR_NUMERIC when its first
    macro step ends; the solves batched with it finish with the same bits as
    alone."""
    from forestclaw_b200.serve import DONE, FAILED, Server

    good = [_dam(seed=30 + k, maxlevel=3 + k, subcycle=1) for k in range(2)]
    alone = [_serve([r])[0] for r in good]
    bad_cfg = _dam_cfg(seed=32, maxlevel=3, subcycle=1)
    bad = cases.to_options(cases.replace(bad_cfg, pparams=tuple(bad_cfg.pparams[:4]) + (-1.0,)))
    sv = Server(1 << 40)
    ids = [sv.submit(good[0]), sv.submit(bad), sv.submit(good[1])]
    sv.run_until_idle()
    assert sv.status(ids[1]).state == FAILED
    assert "NaN" in sv.error(ids[1])
    for k, i in ((0, ids[0]), (1, ids[2])):
        assert sv.status(i).state == DONE
        assert np.array_equal(sv.get_q(i), alone[k])
    sv.close()
