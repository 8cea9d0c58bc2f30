"""Shallow water over bathymetry with the GeoClaw f-wave solver (rpn2_geoclaw +
clawpack46_flux2fw) on the CUDA path against the oracle.

The bathymetry b = -1 + 0.8 exp(-r^2/0.02) comes from exp(), whose last bit
may differ between CUDA and glibc, so states are compared to 1e-12 relative
max-norm (the contract's per-step bound); the lake at rest is checked to
round-off on the patches that the boundary extrapolation does not reach.
"""
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


def _rel_err(a, b):
    return float(np.max(np.abs(a - b))) / max(1.0, float(np.max(np.abs(b))))


def _central_patches(leaves, level):
    """Patches of a uniform level two or more patches away from the domain
    boundary (beyond the reach of the boundary extrapolation in 10 steps)."""
    n = 1 << level
    out = []
    for k, (lv, x, y) in enumerate(leaves):
        ix, iy = x >> (28 - lv), y >> (28 - lv)
        if 2 <= ix <= n - 3 and 2 <= iy <= n - 3:
            out.append(k)
    return out


@pytest.mark.parametrize("mx", [16, 32])
def test_geoclaw_pulse_against_oracle(gpu_lib, mx):
    cfg = cases.bathy_lake(level=2, mx=mx, seed=1)
    dt = 0.5 / (mx * 4)
    o, d = _pair(cfg)
    assert _rel_err(d.get_q(), o.all_q()) <= REL_TOL
    t = 0.0
    for step in range(20):
        c_o = o.advance(t, dt)
        c_d = d.advance_all_levels(t, dt)
        t += dt
        assert _rel_err(d.get_q(), o.all_q()) <= REL_TOL, f"step {step}"
        assert abs(c_d - c_o) <= 1e-12 * c_o


def test_geoclaw_lake_at_rest_is_preserved(gpu_lib):
    cfg = cases.bathy_lake(level=3, mx=16, amp=0.0)
    o, d = _pair(cfg)
    q0 = d.get_q()
    dt = 0.5 / (16 * 8)
    for k in range(10):
        d.advance_all_levels(k * dt, dt)
    inner = _central_patches(d.leaves(), 3)
    assert len(inner) == 16
    dq = np.abs(d.get_q() - q0)[inner][:, :, 2:-2, 2:-2]
    assert float(dq.max()) <= 1e-14, f"lake-at-rest residual {dq.max():.3e}"


def test_geoclaw_amr_macro_steps(gpu_lib):
    cfg = cases.bathy_lake(minlevel=2, maxlevel=4, mx=16, seed=2, amp=0.05)
    o, d = _pair(cfg)
    assert d.leaves() == o.leaves()
    t, dt = 0.0, 0.5 / (16 * 4)
    for k in range(3):
        c_o = o.advance(t, dt)
        c_d = d.advance_all_levels(t, dt)
        assert abs(c_d - c_o) <= 1e-12 * c_o
        t += dt
        assert _rel_err(d.get_q(), o.all_q()) <= REL_TOL, f"macro step {k}"
        o.regrid()
        d.regrid()
        assert d.leaves() == o.leaves()
        assert _rel_err(d.get_q(), o.all_q()) <= REL_TOL, f"after regrid {k}"


def test_geoclaw_rejects_transverse_order(gpu_lib):
    import forestclaw_b200 as fcb

    base = cases.to_options(cases.bathy_lake(level=1, mx=8))
    for kw in ({"order": (2, 2)}, {"claw_version": 5}, {"maux": 0}, {"step_variant": 1}):
        o = cases.to_options(cases.bathy_lake(level=1, mx=8))
        for k, v in kw.items():
            setattr(o, k, v)
        with pytest.raises(fcb.FcbError) as e:
            fcb.Solver(o)
        assert e.value.code == 1, kw
    fcb.Solver(base).close()
