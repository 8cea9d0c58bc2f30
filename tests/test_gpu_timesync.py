"""Conservative time synchronisation (time-sync = T) on the CUDA path.

The registers are accumulated by the step kernel (the four-barrier form, or
the pipelined form, the one that carries the clawpack 5 update) and a
store-flux kernel, the same-size and fine-to-coarse corrections run as
per-patch records; all of it compiled without FMA contraction in the
reference's operation order, so the solution is compared with the oracle bit
for bit, and the reference's radialdam regression runs (cellave2 initial depth
on [-2.5, 2.5]^2, gradient tagging, time-sync; clawpack 4.6 and 5) must give
their pinned counters.
"""
import dataclasses
import json
from pathlib import Path

import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu

PINS = json.loads((Path(__file__).parent / "golden" / "regression_pins.json").read_text())


def _pair(cfg, **extra):
    import forestclaw_b200 as fcb

    opts = cases.to_options(cfg)
    for k, v in extra.items():
        setattr(opts, k, v)
    o = O.OracleSolver(cfg)
    d = fcb.Solver(opts)
    o.initialize()
    d.initialize()
    return o, d


def _oq(o):
    """Oracle patch arrays in the order fcb_get_q returns: (patch, m, j, i) for
    clawpack 4.6, (patch, j, i, m) for clawpack 5."""
    q = o.all_q()
    return np.moveaxis(q, 1, -1) if o.cfg.claw_version == 5 else q


def _fixed_mesh_dam(time_sync=1, claw_version=4, **kw):
    return dataclasses.replace(O.radialdam_regression(claw_version), time_sync=time_sync, regrid_interval=0,
                               minlevel=2, maxlevel=4, **kw)


# (clawpack version, step form): the four-barrier form (1), the pipelined form
# (3), the autotuner's pick between them (0); clawpack 5 runs the pipelined form
FORMS = [(4, 1), (4, 3), (4, 0), (5, 3)]


def test_cellave_initial_depth_bit_exact(gpu_lib):
    o, d = _pair(dataclasses.replace(O.radialdam_regression(), minlevel=3, maxlevel=3))
    assert np.array_equal(d.get_q(), _oq(o))


@pytest.mark.parametrize("claw,form", FORMS)
def test_time_sync_macro_steps_bit_exact_on_fixed_mesh(gpu_lib, claw, form):
    """Subcycled levels 2-4 with intermediate and final synchronisations; the
    waves cross the coarse/fine faces within these steps."""
    o, d = _pair(_fixed_mesh_dam(claw_version=claw), step_variant=form)
    assert d.leaves() == o.leaves()
    assert np.array_equal(d.get_q(), _oq(o))
    t, dt = 0.0, 0.02
    for k in range(12):
        c_o = o.advance(t, dt)
        c_d = d.advance_all_levels(t, dt)
        assert c_d == c_o
        qd, qo = d.get_q(), _oq(o)
        assert np.array_equal(qd, qo), f"macro step {k}: max diff {np.max(np.abs(qd - qo)):.3e}"
        t += dt


@pytest.mark.parametrize("claw,form", [(4, 0), (5, 3)])
def test_time_sync_with_regrid_bit_exact(gpu_lib, claw, form):
    cfg = dataclasses.replace(O.radialdam_regression(claw), minlevel=2, maxlevel=4)
    o, d = _pair(cfg, step_variant=form)
    assert d.leaves() == o.leaves()
    t, dt = 0.0, 0.02
    for k in range(6):
        assert o.advance(t, dt) == d.advance_all_levels(t, dt)
        assert np.array_equal(d.get_q(), _oq(o)), f"macro step {k}"
        t += dt
        o.regrid()
        d.regrid()
        assert d.leaves() == o.leaves()
        assert np.array_equal(d.get_q(), _oq(o)), f"after regrid {k}"


@pytest.mark.parametrize("claw,form", FORMS)
def test_time_sync_conserves_mass_exactly_on_gpu(gpu_lib, claw, form):
    import forestclaw_b200 as fcb

    opts = cases.to_options(dataclasses.replace(_fixed_mesh_dam(claw_version=claw), tfinal=0.3))
    opts.step_variant = form
    d = fcb.Solver(opts)
    d.initialize()
    m0 = d.conservation_check()
    d.run()
    assert d.conservation_check()[0] == m0[0]


@pytest.mark.parametrize("name,claw", [("radialdam", 4), ("radialdam_claw5", 5)])
def test_radialdam_regression_pin_on_gpu(gpu_lib, name, claw):
    """regression_values_0.csv / _1.csv of radialdam (--user:claw-version=4 / 5,
    time-sync = T): the pinned counters, and the final fields equal to the
    oracle's bit for bit."""
    import forestclaw_b200 as fcb

    cfg = O.radialdam_regression(claw)
    d = fcb.Solver(cases.to_options(cfg))
    d.initialize()
    d.run()
    c = d.counters()
    want = PINS[name]["values"]
    assert c["count_amr_advance"] == want["count_amr_advance"]
    assert d.num_patches == want["global_num_patches"]
    assert c["count_amr_new_domain"] == want["count_amr_new_domain"]
    o = O.OracleSolver(cfg, parallel=True)
    o.initialize()
    o.run()
    assert d.leaves() == o.leaves()
    assert np.array_equal(d.get_q(), _oq(o))


def test_time_sync_graph_replay_bit_exact(gpu_lib):
    """The macro-step graph carries the store-flux launches and the
    synchronisation records like every other launch of the schedule."""
    import forestclaw_b200 as fcb

    cfg = _fixed_mesh_dam()
    solvers = []
    for g in (0, 1):
        opts = cases.to_options(cfg)
        opts.macro_graph = g
        s = fcb.Solver(opts)
        s.initialize()
        solvers.append(s)
    t, dt = 0.0, 0.02
    for k in range(5):
        c0 = solvers[0].advance_all_levels(t, dt)
        c1 = solvers[1].advance_all_levels(t, dt)
        assert c0 == c1
        assert np.array_equal(solvers[0].get_q(), solvers[1].get_q()), f"macro step {k}"
        t += dt
    assert solvers[1].counters()["count_graph_replays"] == 3


def test_time_sync_option_checks(gpu_lib):
    import forestclaw_b200 as fcb

    for kw in ({"step_variant": 2}, {"step_variant": 4}, {"precision": fcb.PRECISION_MIXED},
               {"claw_version": 5, "step_variant": 1}):
        opts = cases.to_options(_fixed_mesh_dam())
        for k, v in kw.items():
            setattr(opts, k, v)
        with pytest.raises(fcb.FcbError) as e:
            fcb.Solver(opts)
        assert e.value.code == 1, kw
    opts = cases.to_options(cases.swirl_uniform(level=2))
    opts.time_sync = 1
    with pytest.raises(fcb.FcbError):
        fcb.Solver(opts)
