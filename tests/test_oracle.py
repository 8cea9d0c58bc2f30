"""CPU checks of the oracle itself: the reference's regression pins and
known-answer properties of the method.  No GPU is needed."""
import json
from pathlib import Path

import numpy as np
import pytest

import cases
import oracle as O

PINS = json.loads((Path(__file__).parent / "golden" / "regression_pins.json").read_text())


@pytest.mark.parametrize("name", ["swirl", "quadrants"])
def test_regression_pins(name):
    """applications/**/regression_values_0.csv: count_amr_advance,
    global_num_patches and count_amr_new_domain of the clawpack 4.6 runs."""
    cfg = O.swirl_regression() if name == "swirl" else O.quadrants_regression()
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
