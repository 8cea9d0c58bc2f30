"""CPU checks of the oracle itself: the reference's regression pins and
known-answer properties of the method.  No GPU is needed."""
import json
from pathlib import Path

import numpy as np
import pytest

import cases
import oracle as O

PINS = json.loads((Path(__file__).parent / "golden" / "regression_pins.json").read_text())


PIN_CONFIGS = {
    "swirl": O.swirl_regression, "swirl_claw5": lambda: O.swirl_regression(5),
    "quadrants": O.quadrants_regression, "quadrants_claw5": lambda: O.quadrants_regression(5),
    "radialdam": O.radialdam_regression, "radialdam_claw5": lambda: O.radialdam_regression(5),
    "bump": O.bump_regression, "bump_claw5": lambda: O.bump_regression(5),
    "periodic": O.periodic_regression, "periodic_claw5": lambda: O.periodic_regression(5),
    "filament": O.filament_regression, "filament_claw5": lambda: O.filament_regression(5),
}


@pytest.mark.parametrize("name", sorted(PIN_CONFIGS))
def test_regression_pins(name):
    """applications/**/regression_values_{0,1}.csv: count_amr_advance,
    global_num_patches and count_amr_new_domain of the clawpack 4.6 runs and
    the --user:claw-version=5 runs of swirl, quadrants, bump, the periodic
    brick and the cart-mapped filament brick with capacity (bump's
    clawpack 5 run has solid walls on all four sides, 14 new domains in 24
    advances), and of the radialdam runs with clawpack 4.6 and 5 (time-sync,
    cellave2 initial depth, gradient tagging on [-2.5, 2.5]^2)."""
    cfg = PIN_CONFIGS[name]()
    s = O.OracleSolver(cfg)
    s.initialize()
    s.run()
    c = s.counters()
    want = PINS[name]["values"]
    assert c["count_amr_advance"] == want["count_amr_advance"]
    assert s.num_patches == want["global_num_patches"]
    assert c["count_amr_new_domain"] == want["count_amr_new_domain"]


def test_lake_at_rest_is_exact():
    cfg = cases.radialdam_uniform(level=2, mx=8, hin=1.0, hout=1.0)
    s = O.OracleSolver(cfg)
    s.initialize()
    q0 = s.all_q()
    for k in range(5):
        s.advance(k * 0.01, 0.01)
    assert np.array_equal(s.all_q(), q0)


def test_interior_mass_conservation():
    """A dam break that has not reached the boundary conserves h to round-off."""
    cfg = cases.radialdam_uniform(level=3, mx=16, r0=0.1)
    s = O.OracleSolver(cfg)
    s.initialize()
    m0 = s.conservation()[0]
    for k in range(10):
        s.advance(k * 0.002, 0.002)
    m1 = s.conservation()[0]
    assert abs(m1 - m0) <= 1e-13 * m0


def test_step_is_translation_invariant():
    """Two identical patches at different places give identical updates
    (the SWE step does not depend on position)."""
    cfg = cases.radialdam_uniform(level=0, mx=8)
    rng = np.random.default_rng(1)
    q = np.empty((3, cfg.ny, cfg.nx))
    q[0] = 1.0 + 0.1 * rng.random((cfg.ny, cfg.nx))
    q[1] = 0.05 * rng.standard_normal((cfg.ny, cfg.nx))
    q[2] = 0.05 * rng.standard_normal((cfg.ny, cfg.nx))
    a, b = q.copy(), q.copy()
    ca = O.step2(cfg, a, None, 0.1, 0.1, 0.02)
    cb = O.step2(cfg, b, None, 0.1, 0.1, 0.02)
    assert ca == cb and np.array_equal(a, b)


def test_first_order_upwind_known_answer():
    """order (1,0), constant positive velocity u, v = 0 on one patch: the
    interior update is q_i - (dt/dx) u (q_i - q_{i-1})."""
    cfg = cases.swirl_uniform(level=0, mx=8)
    cfg = cases.replace(cfg, order=(1, 0), mthlim=(0,))
    rng = np.random.default_rng(2)
    q = rng.random((1, cfg.ny, cfg.nx))
    aux = np.zeros((2, cfg.ny, cfg.nx))
    aux[0] = 0.7  # u at the left edge of each cell
    dx = dy = 1.0 / 8
    dt = 0.1
    qn = q.copy()
    O.step2(cfg, qn, aux, dx, dy, dt)
    expect = q[0, :, 1:-1] - dt / dx * 0.7 * (q[0, :, 1:-1] - q[0, :, :-2])
    assert np.allclose(qn[0, 1:-1, 1:-1], expect[1:-1, :], rtol=0, atol=1e-15)


def test_claw5_step_updates_interior_cells_only():
    """clawpack5_step2_wrap.f updates i,j = 1..mx only; clawpack46 also updates
    the ghost band 1-mbc..mx+mbc-1."""
    cfg4 = cases.radialdam_uniform(level=0, mx=8)
    cfg5 = cases.replace(cfg4, claw_version=5)
    s = O.OracleSolver(cfg4)
    s.initialize()
    rng = np.random.default_rng(0)
    qin = s.all_q()[0] + 0.01 * rng.uniform(size=s.all_q()[0].shape)
    qin[0] = np.abs(qin[0]) + 0.5
    q4, q5 = qin.copy(), qin.copy()
    O.step2(cfg4, q4, None, 1 / 8, 1 / 8, 0.01)
    O.step2(cfg5, q5, None, 1 / 8, 1 / 8, 0.01)
    mbc = cfg4.mbc
    ghost = np.ones(qin.shape[1:], bool)
    ghost[mbc:-mbc, mbc:-mbc] = False
    assert np.array_equal(q5[:, ghost], qin[:, ghost])
    assert not np.array_equal(q4[:, ghost], qin[:, ghost])
    assert not np.array_equal(q5[:, ~ghost], qin[:, ~ghost])


def test_claw5_interior_mass_conservation():
    cfg = cases.replace(cases.radialdam_uniform(level=3, mx=16, r0=0.1), claw_version=5)
    s = O.OracleSolver(cfg)
    s.initialize()
    m0 = s.conservation()[0]
    for k in range(10):
        s.advance(k * 0.002, 0.002)
    assert abs(s.conservation()[0] - m0) <= 1e-13 * m0


def test_geoclaw_lake_at_rest_oracle():
    """rpn2_geoclaw's steady-state wave keeps a lake at rest over the bump to
    round-off on patches the boundary extrapolation has not reached."""
    cfg = cases.bathy_lake(level=3, mx=8, amp=0.0)
    s = O.OracleSolver(cfg)
    s.initialize()
    q0 = s.all_q()
    dt = 0.5 / (8 * 8)
    for k in range(6):
        s.advance(k * dt, dt)
    central = [k for k, (lv, x, y) in enumerate(s.leaves())
               if 2 <= x >> 25 <= 5 and 2 <= y >> 25 <= 5]
    assert len(central) == 16
    dq = np.abs(s.all_q() - q0)[central][:, :, 2:-2, 2:-2]
    assert float(dq.max()) <= 1e-14


def test_geoclaw_rejects_transverse_order():
    cfg = cases.replace(cases.bathy_lake(level=1, mx=8), order=(2, 2))
    s = O.OracleSolver(cfg)
    with pytest.raises(Exception):
        s.initialize()
        s.advance(0.0, 0.001)


def _fixed_mesh_dam(time_sync):
    """The radialdam regression case on a mesh refined once at start and never
    regridded, so the waves cross coarse/fine faces (levels 2-4, to t = 0.6)."""
    import dataclasses

    return dataclasses.replace(O.radialdam_regression(), time_sync=time_sync, tfinal=0.6,
                               regrid_interval=0, minlevel=2, maxlevel=4)


def test_time_sync_conserves_mass_exactly():
    """fclaw2d_time_sync's corrections make subcycled AMR conservative: with
    time-sync the Kahan mass sum is unchanged to the last bit while waves cross
    the coarse/fine faces; without it the mass drifts."""
    out = {}
    for ts in (0, 1):
        s = O.OracleSolver(_fixed_mesh_dam(ts))
        s.initialize()
        m0 = s.conservation()
        s.run()
        out[ts] = (m0, s.conservation())
    m0, m1 = out[1]
    assert m1[0] == m0[0]
    m0, m1 = out[0]
    assert abs(m1[0] - m0[0]) > 1e-6 * m0[0]


def test_cellave_initial_depth():
    """cellave2: a cell wholly inside the circle gets hin, wholly outside hout,
    and the volume of the dam equals hin*pi*r0^2 + hout*(area - pi*r0^2) to the
    accuracy of the polygonal cut of each boundary cell."""
    import dataclasses

    cfg = dataclasses.replace(O.radialdam_regression(), minlevel=3, maxlevel=3)
    s = O.OracleSolver(cfg)
    s.initialize()
    q = s.all_q()
    h = q[:, 0, 2:-2, 2:-2]
    assert h.min() == 1.0 and h.max() == 2.0
    assert ((h > 1.0) & (h < 2.0)).any()
    mass = s.conservation()[0]
    exact = 2.0 * np.pi * 0.25 + 1.0 * (25.0 - np.pi * 0.25)
    assert abs(mass - exact) < 1e-3 * exact


def test_time_sync_rejected_outside_its_scope():
    import dataclasses

    for kw in ({"solver": O.EULER4_ROE, "meqn": 4, "mwaves": 4},):
        cfg = dataclasses.replace(_fixed_mesh_dam(1), tfinal=0.01, **kw)
        s = O.OracleSolver(cfg)
        with pytest.raises(Exception):
            s.initialize()
            s.run()


def test_src2_axisymmetric_restates_the_fortran():
    """The oracle's src2 (shockbubble user_4.6/src2.f) against a NumPy
    evaluation of the same formulas with the Fortran association
    (a*b/c*d = ((a*b)/c)*d, rho*u*v = (rho*u)*v), bit for bit, on random
    states; a state with v = 0 is left unchanged."""
    rng = np.random.default_rng(3)
    mbc, mx, gamma1, dt, ylower, dy = 2, 8, 0.4, 1e-3, 0.25, 1.0 / 64
    q = np.empty((5, mx + 4, mx + 4))
    q[0] = rng.uniform(0.5, 2.0, q[0].shape)
    q[1] = rng.uniform(-1.0, 1.0, q[0].shape)
    q[2] = rng.uniform(-1.0, 1.0, q[0].shape)
    q[3] = rng.uniform(2.0, 5.0, q[0].shape)
    q[4] = rng.uniform(0.0, 1.0, q[0].shape)
    want = q.copy()
    dt2 = dt / 2.0
    for j in range(1, mx + 1):
        for i in range(1, mx + 1):
            jj, ii = j + mbc - 1, i + mbc - 1
            rad = ylower + (j - 0.5) * dy
            q1, q2, q3, q4 = (float(want[m, jj, ii]) for m in range(4))
            rho, u, v = q1, q2 / q1, q3 / q1
            press = gamma1 * (q4 - 0.5 * rho * (u * u + v * v))
            qs1 = q1 - dt2 * 1.0 / rad * q3
            qs2 = q2 - dt2 * 1.0 / rad * (rho * u * v)
            qs3 = q3 - dt2 * 1.0 / rad * (rho * v * v)
            qs4 = q4 - dt2 * 1.0 / rad * v * (q4 + press)
            rho, u, v = qs1, qs2 / qs1, qs3 / qs1
            press = gamma1 * (qs4 - 0.5 * rho * (u * u + v * v))
            want[0, jj, ii] = q1 - dt * 1.0 / rad * qs3
            want[1, jj, ii] = q2 - dt * 1.0 / rad * (rho * u * v)
            want[2, jj, ii] = q3 - dt * 1.0 / rad * (rho * v * v)
            want[3, jj, ii] = q4 - dt * 1.0 / rad * v * (qs4 + press)
    got = q.copy()
    O.src2_axisymmetric(got, mbc, ylower, dy, gamma1, dt)
    assert np.array_equal(got, want)
    assert np.array_equal(got[4], q[4])  # the tracer is not a source component
    still = q.copy()
    still[2] = 0.0
    moved = still.copy()
    O.src2_axisymmetric(moved, mbc, ylower, dy, gamma1, dt)
    assert np.array_equal(moved, still)
