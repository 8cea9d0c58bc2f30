"""Ghost-exchange fusion (ghost_fusion = 2) against the unfused path
(ghost_fusion = 1) and the oracle.

On a mesh of one level the fused step reads its ghost cells from the
neighbours' interiors (the values the same-size copies and the physical
boundary conditions would write), writes the updated interiors into a second
arena, and the last ghost update of a macro step waits until something reads
ghost cells.  Every array a caller sees must equal the unfused path's bit for
bit (and the oracle's within the tolerances of the other parity tests: exact
for the Roe and f-wave solvers apart from exp() in the bathymetry, 1e-12 for
the swirl velocities from sin()).
"""
import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu


def _rel_err(a, b):
    return float(np.max(np.abs(a - b))) / max(1.0, float(np.max(np.abs(b))))


def _oracle_q(o):
    q = o.all_q()
    return np.moveaxis(q, 1, -1) if o.cfg.claw_version == 5 else q


def _solver(cfg, fusion, **extra):
    import forestclaw_b200 as fcb

    opts = cases.to_options(cfg)
    opts.ghost_fusion = fusion
    for k, v in extra.items():
        setattr(opts, k, v)
    d = fcb.Solver(opts)
    d.initialize()
    return d


CASES = {
    "swirl8": (lambda: cases.swirl_uniform(level=3, mx=8), lambda: cases.swirl_dt(level=3, mx=8), 1e-12),
    "swirl16": (lambda: cases.swirl_uniform(level=3, mx=16), lambda: cases.swirl_dt(level=3, mx=16), 1e-12),
    "swirl32": (lambda: cases.swirl_uniform(level=2, mx=32), lambda: cases.swirl_dt(level=2, mx=32), 1e-12),
    "dam_walls": (lambda: cases.replace(cases.radialdam_uniform(level=2, mx=16), mthbc=(3, 3, 3, 3),
                                        pparams=(0.3, 0.65, 0.2, 2.0, 1.0)), lambda: 0.4 / 64 / 1.5, 0.0),
    "dam_mixed_bc": (lambda: cases.replace(cases.radialdam_uniform(level=2, mx=32), mthbc=(3, 1, 1, 3),
                                           pparams=(0.3, 0.65, 0.2, 2.0, 1.0)), lambda: 0.4 / 128 / 1.5, 0.0),
    "quadrants": (lambda: cases.quadrants_uniform(level=2, mx=16), lambda: 0.3 / 64 / 2.0, 0.0),
    "claw5_dam": (lambda: cases.replace(cases.radialdam_uniform(level=2, mx=16), claw_version=5, mthbc=(1, 3, 3, 1),
                                        pparams=(0.3, 0.65, 0.2, 2.0, 1.0)), lambda: 0.4 / 64 / 1.5, 0.0),
    "claw5_swirl": (lambda: cases.replace(cases.swirl_uniform(level=3, mx=16), claw_version=5),
                    lambda: cases.swirl_dt(level=3, mx=16), 1e-12),
    "geoclaw": (lambda: cases.bathy_lake(level=3, mx=16, seed=2, amp=0.05), lambda: 0.5 / (16 * 8), 1e-12),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_fused_steps_equal_unfused_and_oracle(gpu_lib, name):
    """Fused and unfused solves, compared after every step (each read runs the
    deferred ghost update) and after five steps in a row with no read between
    them (the fused steps then never run a ghost fill)."""
    make_cfg, make_dt, tol = CASES[name]
    cfg, dt = make_cfg(), make_dt()
    o = O.OracleSolver(cfg)
    o.initialize()
    fused, plain = _solver(cfg, 2), _solver(cfg, 1)
    t = 0.0
    for k in range(4):
        c_o = o.advance(t, dt)
        c_f = fused.advance_all_levels(t, dt)
        c_p = plain.advance_all_levels(t, dt)
        t += dt
        assert c_f == c_p, (k, c_f, c_p)
        assert abs(c_f - c_o) <= tol * max(1.0, c_o)
        qf = fused.get_q()
        assert np.array_equal(qf, plain.get_q()), f"step {k}"
        assert _rel_err(qf, _oracle_q(o)) <= tol, f"step {k}"
    waves0 = fused.counters()["count_ghost_waves"]
    for k in range(5):
        o.advance(t, dt)
        fused.advance_all_levels(t, dt)
        plain.advance_all_levels(t, dt)
        t += dt
    assert fused.counters()["count_ghost_waves"] == waves0  # no fill ran between the fused steps
    qf = fused.get_q()
    assert np.array_equal(qf, plain.get_q())
    assert _rel_err(qf, _oracle_q(o)) <= tol
    ms, f = fused.step_kernel_time(t, dt, 2)
    assert f and ms > 0.0
    ms, f = plain.step_kernel_time(t, dt, 2)
    assert not f and ms > 0.0


def test_fused_mixed_precision_equals_unfused_mixed(gpu_lib):
    """The fused mixed form has the unfused mixed form's arithmetic."""
    import forestclaw_b200 as fcb

    cfg = cases.swirl_uniform(level=4, mx=16)
    dt = cases.swirl_dt(level=4, mx=16)
    fused = _solver(cfg, 2, precision=fcb.PRECISION_MIXED)
    plain = _solver(cfg, 1, precision=fcb.PRECISION_MIXED)
    t = 0.0
    for _ in range(10):
        assert fused.advance_all_levels(t, dt) == plain.advance_all_levels(t, dt)
        t += dt
    assert np.array_equal(fused.get_q(), plain.get_q())


@pytest.mark.parametrize("subcycle", [1, 0])
def test_fused_single_level_above_minlevel(gpu_lib, subcycle):
    """A mesh refined everywhere to maxlevel = minlevel + 1 (value criterion
    with threshold 0): the macro step is two fine steps of dt/2 with a ghost
    update between them (subcycled, or non-subcycled with rf = 2)."""
    cfg = cases.replace(cases.radialdam_amr(seed=0, minlevel=2, maxlevel=3, mx=16), criteria=O.VALUE,
                        refine_threshold=0.0, coarsen_threshold=0.0, regrid_interval=0, subcycle=subcycle)
    o = O.OracleSolver(cfg)
    o.initialize()
    assert {lv for lv, _, _ in o.leaves()} == {3}
    fused, plain = _solver(cfg, 2), _solver(cfg, 1)
    assert fused.leaves() == o.leaves()
    t, dt = 0.0, cfg.initial_dt
    for k in range(3):
        c_o = o.advance(t, dt)
        assert fused.advance_all_levels(t, dt) == c_o
        assert plain.advance_all_levels(t, dt) == c_o
        t += dt
    q = o.all_q()
    assert np.array_equal(fused.get_q(), q)
    assert np.array_equal(plain.get_q(), q)
    c_f, c_p = fused.counters(), plain.counters()
    assert c_f["count_single_step"] == c_p["count_single_step"]


def test_fused_run_with_cfl_retry(gpu_lib):
    """fcb_run with adaptive dt on a uniform mesh, no regrid, and an initial dt
    that gives CFL 1.27 on the first macro step: it is rejected and restores
    the saved state, whose ghost cells still wait for the deferred update; the
    run equals the unfused run and the oracle bit for bit."""
    base = cases.radialdam_uniform(level=3, mx=16)
    cfg = cases.replace(base, use_fixed_dt=0, regrid_interval=0, tfinal=0.03, max_cfl=1.0, desired_cfl=0.9,
                        initial_dt=0.9 / (16 * 8))
    probe = O.OracleSolver(cfg)
    probe.initialize()
    assert probe.advance(0.0, cfg.initial_dt) > 1.0  # the first try is rejected
    assert np.isfinite(probe.all_q()).all()
    o = O.OracleSolver(cfg)
    o.initialize()
    o.run()
    fused, plain = _solver(cfg, 2), _solver(cfg, 1)
    fused.run()
    plain.run()
    co, cf, cp = o.counters(), fused.counters(), plain.counters()
    assert cf["count_amr_advance"] == cp["count_amr_advance"] == co["count_amr_advance"]
    assert cf["count_single_step"] == co["count_single_step"]
    q = o.all_q()
    assert np.array_equal(fused.get_q(), q)
    assert np.array_equal(plain.get_q(), q)


def test_fused_steps_interleaved_with_other_calls(gpu_lib):
    """Fused advances mixed with a level update, an explicit ghost update, a
    physical-boundary fill and set_q: each of those first runs the deferred
    ghost update (set_q instead overwrites every cell), so both solves stay
    identical."""
    cfg = cases.replace(cases.radialdam_uniform(level=2, mx=16), mthbc=(3, 1, 3, 1),
                        pparams=(0.35, 0.6, 0.2, 2.0, 1.0))
    dt = 0.4 / 64 / 1.5
    fused, plain = _solver(cfg, 2), _solver(cfg, 1)
    t = 0.0

    def both(fn):
        return fn(fused), fn(plain)

    for k in range(2):
        a, b = both(lambda s: s.advance_all_levels(t, dt))
        assert a == b
        t += dt
    a, b = both(lambda s: s.update_single_step(2, t, dt))  # reads ghost cells: the fill runs first
    assert a == b
    assert np.array_equal(fused.get_q(), plain.get_q())
    both(lambda s: s.ghost_update(2, 2, t, 0))
    a, b = both(lambda s: s.advance_all_levels(t, dt))
    assert a == b
    t += dt
    both(lambda s: s.physical_set_bc(2, 0))
    a, b = both(lambda s: s.advance_all_levels(t, dt))
    assert a == b
    t += dt
    q = plain.get_q()
    q[..., 2:-2, 2:-2] *= 1.01
    both(lambda s: s.set_q(q))
    for k in range(2):
        a, b = both(lambda s: s.advance_all_levels(t, dt))
        assert a == b
        t += dt
    assert np.array_equal(fused.get_q(), plain.get_q())
    assert np.array_equal(fused.conservation_check(), plain.conservation_check())


def test_autotuned_fusion_is_bit_identical(gpu_lib):
    """ghost_fusion = 0 lets the tuner time the fused step against the best
    unfused form plus the ghost fill; whichever it picks, the result is the
    unfused one."""
    cfg = cases.swirl_uniform(level=5, mx=16)
    dt = cases.swirl_dt(level=5, mx=16)
    auto, plain = _solver(cfg, 0), _solver(cfg, 1)
    t = 0.0
    for _ in range(4):
        assert auto.advance_all_levels(t, dt) == plain.advance_all_levels(t, dt)
        t += dt
    assert np.array_equal(auto.get_q(), plain.get_q())


def test_fusion_stays_off_on_multilevel_meshes(gpu_lib):
    """On a mesh of several levels the ghost updates include averages,
    interpolations and time interpolation: the fused path is not used."""
    cfg = cases.quadrants_amr(seed=1, minlevel=2, maxlevel=5, mx=8)  # leaves on levels 4 and 5
    d = _solver(cfg, 2)
    assert len({lv for lv, _, _ in d.leaves()}) > 1
    ms, f = d.step_kernel_time(0.0, cfg.initial_dt, 2)
    assert not f and ms > 0.0
