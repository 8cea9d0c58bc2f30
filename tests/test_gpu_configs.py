"""The CUDA path against the oracle at the sizes of the benchmarked
configurations, and the method options the smaller parity tests leave out.

* the plain-method advection case as stated: uniform level 4, mx = 16, 200
  steps, every step within 1e-12 relative max-norm (the swirl velocities come
  from sin(), whose last bit may differ between CUDA and glibc);
* AMR shallow water: levels 3-6, mx = 32, seeds 0 and 1, three macro steps
  with a regrid after each, bit for bit;
* AMR Euler: levels 2-7, mx = 16 and 64, two macro steps, bit for bit;
* shallow water over bathymetry: levels 4-7, mx = 32, two macro steps (the
  bathymetry comes from exp(): 1e-12);
* the non-subcycled schedule (fclaw2d_advance.c:300-324), which every served
  solve runs; solid walls (mthbc = 3); the limiters 1, 2, 3, 5 and 6 of
  clawpack46_inlinelimiter.f (clawpack 5 has 1-5); the "value" refinement
  criterion; and the CFL rejection of fclaw2d_run.c:227-231 (restore the saved
  step, shrink dt, retry).

The large configurations use the OpenMP build of the oracle (the same
arithmetic and compiler flags, patches of a level on several threads).
Each macro step's dt follows the run loop's rule dt * desired_cfl / cfl.
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


def _pair(cfg, parallel=False, **extra):
    import forestclaw_b200 as fcb

    opts = cases.to_options(cfg)
    for k, v in extra.items():
        setattr(opts, k, v)
    o = O.OracleSolver(cfg, parallel=parallel)
    d = fcb.Solver(opts)
    o.initialize()
    d.initialize()
    return o, d


def _macro_steps(o, d, nmacro, dt, tol=0.0, regrid=True):
    """advance_all_levels (+ regrid) on both sides, comparing the CFL number,
    the mesh and every patch array after each advance and each regrid."""
    assert d.leaves() == o.leaves()
    assert _rel_err(d.get_q(), _oracle_q(o)) <= tol, "initial state"
    t = 0.0
    levels = set()
    for k in range(nmacro):
        levels |= {lv for lv, _, _ in o.leaves()}
        c_o = o.advance(t, dt)
        c_d = d.advance_all_levels(t, dt)
        if tol == 0.0:
            assert c_d == c_o, (k, c_d, c_o)
        else:
            assert abs(c_d - c_o) <= tol * max(1.0, c_o), (k, c_d, c_o)
        err = _rel_err(d.get_q(), _oracle_q(o))
        assert err <= tol, f"macro step {k}: rel err {err:.3e}"
        t += dt
        if regrid:
            o.regrid()
            d.regrid()
            assert d.leaves() == o.leaves(), f"mesh after regrid {k}"
            err = _rel_err(d.get_q(), _oracle_q(o))
            assert err <= tol, f"after regrid {k}: rel err {err:.3e}"
        dt = dt * o.cfg.desired_cfl / c_o
    return levels


def test_plain_method_case_as_stated(gpu_lib):
    """Scalar advection, clawpack46, FP64, uniform level 4 (256 patches),
    mx = my = 16, MC limiter, order (2,2), swirl velocities, q0 = 1 for x < 0.5,
    CFL 0.9, fixed dt, 200 steps: within 1e-12 after every step."""
    cfg = cases.swirl_uniform(level=4, mx=16)
    dt = cases.swirl_dt(level=4, mx=16)
    o, d = _pair(cfg)
    assert d.num_patches == 256
    assert np.array_equal(d.get_q(), o.all_q())
    t = 0.0
    worst = 0.0
    for step in range(200):
        c_o = o.advance(t, dt)
        c_d = d.advance_all_levels(t, dt)
        t += dt
        err = _rel_err(d.get_q(), o.all_q())
        worst = max(worst, err)
        assert err <= 1e-12, f"step {step}: rel err {err:.3e}"
        assert abs(c_d - c_o) <= 1e-12 * max(1.0, c_o), (step, c_d, c_o)
    m_o, m_d = o.conservation(), d.conservation_check()
    assert abs(m_d[0] - m_o[0]) <= 1e-13 * abs(m_o[0])


@pytest.mark.slow
@pytest.mark.parametrize("seed", [0, 1])
def test_amr_shallow_water_config(gpu_lib, seed):
    """Radial dam break, Roe solver, levels 3-6 subcycled, mx = 32, gradient
    tagging on h with a regrid after every macro step: bit for bit."""
    cfg = cases.radialdam_amr(seed=seed, minlevel=3, maxlevel=6, mx=32)
    o, d = _pair(cfg, parallel=True)
    levels = _macro_steps(o, d, 3, cfg.initial_dt)
    assert max(levels) == 6 and len(levels) >= 3  # smooth refinement lifts every level-3 leaf
    assert o.num_patches > 1000


@pytest.mark.slow
@pytest.mark.parametrize("mx", [16, 64])
def test_amr_euler_config(gpu_lib, mx):
    """Four-quadrant Riemann problem, Euler Roe solver with entropy fix,
    levels 2-7 subcycled (32 fine steps per macro step), density-gradient
    tagging: bit for bit at mx = 16 and 64."""
    cfg = cases.quadrants_amr(seed=0, minlevel=2, maxlevel=7, mx=mx)
    o, d = _pair(cfg, parallel=True)
    levels = _macro_steps(o, d, 2, cfg.initial_dt)
    assert max(levels) == 7 and len(levels) >= 3


@pytest.mark.slow
def test_bathymetry_config(gpu_lib):
    """GeoClaw f-waves over the Gaussian bump with a surface pulse, levels 4-7,
    mx = 32, a regrid after each macro step."""
    cfg = cases.bathy_lake(level=4, mx=32, seed=0, minlevel=4, maxlevel=7)
    o, d = _pair(cfg, parallel=True)
    levels = _macro_steps(o, d, 2, 0.9 / (32 * 16) / 2, tol=1e-12)
    assert max(levels) == 7


@pytest.mark.parametrize("solver", ["radialdam", "quadrants", "swirl"])
def test_non_subcycled_schedule(gpu_lib, solver):
    """subcycle = 0: every level takes 2^(maxlevel-minlevel) steps of dt/rf with
    ghost updates between them (fclaw2d_advance.c:300-324); served solves run
    this schedule."""
    if solver == "radialdam":
        cfg = cases.replace(cases.radialdam_amr(seed=0, minlevel=3, maxlevel=5, mx=16), subcycle=0)
        dt, tol = cfg.initial_dt, 0.0
    elif solver == "quadrants":
        cfg = cases.replace(cases.quadrants_amr(seed=1, minlevel=2, maxlevel=5, mx=8), subcycle=0)
        dt, tol = cfg.initial_dt, 0.0
    else:
        cfg = cases.replace(O.swirl_regression(), subcycle=0, maxlevel=5)
        dt, tol = cfg.initial_dt, 1e-12
    o, d = _pair(cfg)
    levels = _macro_steps(o, d, 3, dt, tol=tol)
    assert len(levels) >= 2


@pytest.mark.slow
def test_non_subcycled_config_size(gpu_lib):
    """The non-subcycled schedule on the shallow-water configuration
    (levels 3-6, mx = 32): bit for bit."""
    cfg = cases.replace(cases.radialdam_amr(seed=1, minlevel=3, maxlevel=6, mx=32), subcycle=0)
    o, d = _pair(cfg, parallel=True)
    _macro_steps(o, d, 2, cfg.initial_dt)


@pytest.mark.parametrize("variant", [1, 3])
@pytest.mark.parametrize("mthbc", [(3, 3, 3, 3), (3, 1, 1, 3), (1, 3, 3, 1)])
def test_solid_walls_uniform(gpu_lib, mthbc, variant):
    """mthbc = 3 (clawpack46_bc2_default.f: mirror, normal momentum negated) on
    an off-centre dam break whose waves reach the walls: bit for bit."""
    cfg = cases.replace(cases.radialdam_uniform(level=2, mx=16), mthbc=mthbc,
                        pparams=(0.3, 0.65, 0.2, 2.0, 1.0))
    dt = 0.4 / (16 * 4) / 1.5
    o, d = _pair(cfg, step_variant=variant)
    _macro_steps(o, d, 24, dt, regrid=False)


@pytest.mark.parametrize("claw_version", [4, 5])
def test_solid_walls_amr(gpu_lib, claw_version):
    """Walls on an AMR shallow-water solve (coarse and fine patches at the
    walls, clawpack 4.6 and 5): mesh and fields bit for bit."""
    cfg = cases.replace(cases.radialdam_amr(seed=3, minlevel=2, maxlevel=4, mx=16), mthbc=(3, 3, 1, 3),
                        pparams=(0.35, 0.6, 0.22, 2.0, 1.0), claw_version=claw_version)
    o, d = _pair(cfg)
    _macro_steps(o, d, 5, cfg.initial_dt)


@pytest.mark.parametrize("variant", [1, 3])
@pytest.mark.parametrize("limiter", [1, 2, 3, 5, 6])
def test_limiters_shallow_water(gpu_lib, limiter, variant):
    """Minmod (1), superbee (2), van Leer (3), Beam-Warming (5) and the
    generalised minmod with theta = 1.3 (6; a REAL*4 literal in the
    reference): bit for bit in both step forms."""
    cfg = cases.replace(cases.radialdam_uniform(level=2, mx=16), mthlim=(limiter,) * 3)
    o, d = _pair(cfg, step_variant=variant)
    _macro_steps(o, d, 8, 0.4 / (16 * 4) / 1.5, regrid=False)


@pytest.mark.parametrize("limiter", [1, 2, 3, 5])
def test_limiters_claw5(gpu_lib, limiter):
    """clawpack5_inlinelimiter.f (limiters 1-5) on the Euler system: bit for bit."""
    cfg = cases.replace(cases.quadrants_uniform(level=2, mx=16), mthlim=(limiter,) * 4, claw_version=5)
    o, d = _pair(cfg)
    _macro_steps(o, d, 6, 0.3 / (16 * 4) / 2.0, regrid=False)


@pytest.mark.parametrize("limiter", [1, 2, 5, 6])
def test_limiters_scalar_advection(gpu_lib, limiter):
    """The pipelined scalar form reads the limiter from its arguments unless
    it is MC or van Leer: limiters 1, 2, 5 and 6 on the swirl case."""
    cfg = cases.replace(cases.swirl_uniform(level=3, mx=16), mthlim=(limiter,))
    o, d = _pair(cfg, step_variant=3)
    _macro_steps(o, d, 10, cases.swirl_dt(level=3, mx=16), tol=1e-12, regrid=False)


def test_value_criterion(gpu_lib):
    """refinement-criteria = value (fclaw2d_clawpatch_value_exceeds_th.f90):
    refine where h exceeds 1.5, coarsen where no cell exceeds 1.05 (a small dam
    without smooth refinement, so the mesh keeps levels 2-4)."""
    import forestclaw_b200 as fcb

    cfg = cases.replace(cases.radialdam_amr(seed=0, minlevel=2, maxlevel=4, mx=16), criteria=O.VALUE,
                        refine_threshold=1.5, coarsen_threshold=1.05, smooth_refine=0,
                        pparams=(0.5, 0.5, 0.12, 2.0, 1.0))
    o, d = _pair(cfg)
    assert fcb.TAG_VALUE == O.VALUE
    levels = _macro_steps(o, d, 5, cfg.initial_dt)
    assert levels == {2, 3, 4}


@pytest.mark.parametrize("claw_version", [4, 5])
def test_cfl_rejection_and_retry(gpu_lib, claw_version):
    """fclaw2d_run outstyle 1 with adaptive dt and an initial dt 1.5 times too
    large: the first macro step reaches CFL 1.67 > max_cfl, the saved state is
    restored (restore_time_step), dt shrinks to dt*desired_cfl/cfl and the step
    is retaken (fclaw2d_run.c:227-231).  The GPU run equals the oracle's bit for
    bit, with the same counters.  (At 1.8 times the rejected step already
    drives depths negative; the library then reports a NaN CFL as
    FCB_ERR_NUMERIC where the reference's MAX of a NaN speed is compiler
    dependent, so the forced rejection stays below that.)"""
    base = cases.radialdam_amr(seed=0, minlevel=2, maxlevel=4, mx=16, tfinal=0.05)
    cfg = cases.replace(base, initial_dt=1.5 * base.initial_dt, claw_version=claw_version)
    probe = O.OracleSolver(cfg)
    probe.initialize()
    assert probe.advance(0.0, cfg.initial_dt) > cfg.max_cfl  # the first try is rejected
    assert np.isfinite(probe.all_q()).all()
    o, d = _pair(cfg)
    o.run()
    d.run()
    co, cd = o.counters(), d.counters()
    for k in ("count_amr_advance", "count_amr_regrid", "count_amr_new_domain", "count_single_step"):
        assert cd[k] == co[k], k
    assert co["count_amr_advance"] - co["count_amr_regrid"] >= 1  # at least one step was retaken
    assert d.leaves() == o.leaves()
    assert np.array_equal(d.get_q(), _oracle_q(o))
    assert d.curr_time == pytest.approx(cfg.tfinal, rel=1e-12)


@pytest.mark.parametrize("variant", [4, 5])
@pytest.mark.parametrize("solver", ["radialdam", "quadrants"])
@pytest.mark.parametrize("mx", [8, 32])
def test_row_bands_uniform(gpu_lib, solver, mx, variant):
    """The four-barrier form with every patch's rows split into 2 (variant 4)
    or 3 (variant 5) bands of separate CTAs: each band starts two rows early,
    reads a copy of the arena and updates its own rows; every array and the
    CFL number bit for bit."""
    if solver == "radialdam":
        cfg, dt = cases.replace(cases.radialdam_uniform(level=2, mx=mx), mthbc=(3, 1, 1, 3),
                                pparams=(0.3, 0.65, 0.2, 2.0, 1.0)), 0.4 / (mx * 4) / 1.5
    else:
        cfg, dt = cases.quadrants_uniform(level=2, mx=mx), 0.3 / (mx * 4) / 2.0
    o, d = _pair(cfg, step_variant=variant)
    _macro_steps(o, d, 6, dt, regrid=False)


@pytest.mark.parametrize("variant", [4, 5])
def test_row_bands_amr_time_interpolation(gpu_lib, variant):
    """Row bands on an AMR shallow-water solve with subcycling: the bands write
    the pre-step copy (qlast) of the patches with finer neighbours row by row,
    which the time interpolation reads; mesh and fields bit for bit through
    regrids."""
    cfg = cases.radialdam_amr(seed=1, minlevel=2, maxlevel=4, mx=16)
    o, d = _pair(cfg, step_variant=variant)
    _macro_steps(o, d, 4, cfg.initial_dt)


def test_row_bands_time_sync_rejected(gpu_lib):
    import forestclaw_b200 as fcb

    opts = cases.to_options(cases.replace(O.radialdam_regression(), time_sync=1))
    opts.step_variant = 4
    with pytest.raises(fcb.FcbError):
        fcb.Solver(opts)


@pytest.mark.parametrize("solver", ["radialdam", "quadrants"])
def test_banded_last_wave(gpu_lib, solver):
    """A level update whose CTAs end with a small last wave: on B200 (148 SMs,
    one four-barrier Roe CTA of 12 patches of mx = 16 per SM) a level of 4,096
    patches is 342 CTAs, two full waves and a tail of 46, which the launcher
    splits into 3 row bands read from a copy of those patches.  Every array
    and the CFL number equal the oracle's bit for bit, through three macro
    steps (ghost updates between them, no regrid)."""
    if solver == "radialdam":
        cfg, dt = cases.replace(cases.radialdam_uniform(level=6, mx=16), mthbc=(3, 1, 1, 3)), 0.4 / (16 * 64) / 1.5
    else:
        cfg, dt = cases.quadrants_uniform(level=6, mx=16), 0.3 / (16 * 64) / 2.0
    o, d = _pair(cfg, parallel=True, step_variant=1)
    _macro_steps(o, d, 3, dt, regrid=False)
