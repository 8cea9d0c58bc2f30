"""The clawpack 5 update (fc2d_clawpack5) on the CUDA path against the oracle.

fc2d_clawpack5 differs from fc2d_clawpack46 in its loop ranges (fluxes at
interfaces 1..mx+1 only, interior cells updated), in the shallow-water Roe
solver's arithmetic (clawpack5_rpn2.f90 / clawpack5_rpt2.f90) and in the
array order q(m,i,j), which fcb_get_q returns for claw_version 5.  The
tolerances are those of the clawpack 4.6 parity tests: bit-exact except for
the swirl velocities, whose sin() may differ in the last bit (1e-12).
"""
import json
from pathlib import Path

import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12


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


def _oracle_q5(o):
    """Oracle patch arrays in the clawpack 5 order (patch, j, i, m)."""
    return np.moveaxis(o.all_q(), 1, -1)


def _rel_err(a, b):
    return float(np.max(np.abs(a - b))) / max(1.0, float(np.max(np.abs(b))))


@pytest.mark.parametrize("mx", [8, 16, 32])
def test_claw5_swirl_uniform(gpu_lib, mx):
    cfg = cases.replace(cases.swirl_uniform(level=3, mx=mx), claw_version=5)
    dt = cases.swirl_dt(level=3, mx=mx)
    o, d = _pair(cfg)
    q0 = d.get_q()
    assert q0.shape[-1] == 1 and q0.shape[1:3] == (cfg.ny, cfg.nx)
    assert np.array_equal(q0, _oracle_q5(o))
    t = 0.0
    for step in range(10):
        c_o = o.advance(t, dt)
        c_d = d.advance_all_levels(t, dt)
        t += dt
        assert _rel_err(d.get_q(), _oracle_q5(o)) <= REL_TOL, f"step {step}"
        assert abs(c_d - c_o) <= 1e-12 * max(1.0, c_o)


@pytest.mark.parametrize("name", ["radialdam", "quadrants"])
def test_claw5_roe_solvers_bit_exact(gpu_lib, name):
    if name == "radialdam":
        cfg = cases.replace(cases.radialdam_uniform(level=2, mx=16), claw_version=5)
        dt = 0.4 / (16 * 4) / 1.5
    else:
        cfg = cases.replace(cases.quadrants_uniform(level=2, mx=16), claw_version=5)
        dt = 0.3 / (16 * 4) / 2.0
    o, d = _pair(cfg)
    t = 0.0
    for step in range(8):
        c_o = o.advance(t, dt)
        c_d = d.advance_all_levels(t, dt)
        t += dt
        qd, qo = d.get_q(), _oracle_q5(o)
        assert np.array_equal(qd, qo), f"step {step}: max diff {np.max(np.abs(qd - qo)):.3e}"
        assert c_d == c_o


def test_claw5_differs_from_claw46(gpu_lib):
    """The two updates are different methods on the same data (interior-only
    update, shallow-water arithmetic), so their states part after a few steps."""
    base = cases.radialdam_uniform(level=2, mx=16)
    dt = 0.4 / (16 * 4) / 1.5
    _, d4 = _pair(base)
    _, d5 = _pair(cases.replace(base, claw_version=5))
    for k in range(3):
        d4.advance_all_levels(k * dt, dt)
        d5.advance_all_levels(k * dt, dt)
    assert not np.array_equal(np.moveaxis(d4.get_q(), 1, -1), d5.get_q())


def test_claw5_set_q_round_trip(gpu_lib):
    cfg = cases.replace(cases.quadrants_uniform(level=1, mx=8), claw_version=5)
    _, d = _pair(cfg)
    rng = np.random.default_rng(3)
    q = rng.uniform(0.5, 1.5, size=d.get_q().shape)
    d.set_q(q)
    assert np.array_equal(d.get_q(), q)


def test_claw5_regression_pin_on_gpu(gpu_lib):
    """regression_values_1.csv (swirl, --user:claw-version=5)."""
    pins = json.loads((Path(__file__).parent / "golden" / "regression_pins.json").read_text())
    want = pins["swirl_claw5"]["values"]
    cfg = O.swirl_regression(5)
    o, d = _pair(cfg)
    o.run()
    d.run()
    c = d.counters()
    assert c["count_amr_advance"] == want["count_amr_advance"]
    assert d.num_patches == want["global_num_patches"]
    assert c["count_amr_new_domain"] == want["count_amr_new_domain"]
    assert d.leaves() == o.leaves()
    assert _rel_err(d.get_q(), _oracle_q5(o)) <= 1e-11


def test_claw5_amr_macro_steps_bit_exact(gpu_lib):
    cfg = cases.replace(cases.radialdam_amr(seed=3, minlevel=2, maxlevel=4, mx=16, tfinal=0.05),
                        claw_version=5)
    o, d = _pair(cfg)
    assert d.leaves() == o.leaves()
    t, dt = 0.0, 0.9 / (16 * 4) / 1.5
    for k in range(3):
        assert d.advance_all_levels(t, dt) == o.advance(t, dt)
        t += dt
        assert np.array_equal(d.get_q(), _oracle_q5(o)), f"macro step {k}"
        o.regrid()
        d.regrid()
        assert d.leaves() == o.leaves()
        assert np.array_equal(d.get_q(), _oracle_q5(o)), f"after regrid {k}"


def test_claw5_mixed_precision(gpu_lib):
    import forestclaw_b200 as fcb

    cfg = cases.replace(cases.radialdam_uniform(level=2, mx=16), claw_version=5)
    dt = 0.4 / (16 * 4) / 1.5
    o, d = _pair(cfg, precision=fcb.PRECISION_MIXED)
    for k in range(20):
        o.advance(k * dt, dt)
        d.advance_all_levels(k * dt, dt)
    a, b = d.get_q()[:, 2:-2, 2:-2, :], _oracle_q5(o)[:, 2:-2, 2:-2, :]
    assert float(np.abs(a - b).sum() / np.abs(b).sum()) <= 1e-5
