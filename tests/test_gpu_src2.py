"""The src2 stage (clawpack46_update / clawpack5_update call src2 after the
step when src_term > 0) on the CUDA path against the oracle: the axisymmetric
Euler source of euler/2d/shockbubble (radius y at the cell centre), with a
solid wall on the axis (mthbc(3) = 3), bit for bit.
"""
import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu


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


def _oracle_q(o):
    q = o.all_q()
    return np.moveaxis(q, 1, -1) if o.cfg.claw_version == 5 else q


@pytest.mark.parametrize("claw_version, variant", [(4, 1), (4, 3), (5, 3)])  # clawpack 5: pipelined form only
def test_src2_uniform(gpu_lib, variant, claw_version):
    # the four quadrant states of euler/2d/quadrants with v = 0, split at (0.5, 0.5):
    # an axisymmetric flow has no velocity across the axis y = 0 (the wall)
    states = [(s[0], s[1], 0.0, s[3]) for s in O.QUADRANT_STATES]
    cfg = cases.replace(cases.quadrants_uniform(level=2, mx=16), src_term=1, mthbc=(1, 1, 3, 1),
                        claw_version=claw_version, pparams=O.quadrants_params(states, 0.5, 0.5))
    dt = 0.3 / 64 / 2.0
    o, d = _pair(cfg, step_variant=variant)
    plain = O.OracleSolver(cases.replace(cfg, src_term=0))
    plain.initialize()
    t = 0.0
    for k in range(8):
        c_o = o.advance(t, dt)
        plain.advance(t, dt)
        assert d.advance_all_levels(t, dt) == c_o
        t += dt
        assert np.array_equal(d.get_q(), _oracle_q(o)), f"step {k}"
    assert not np.array_equal(o.all_q(), plain.all_q())  # the source did change the state


def test_src2_amr_subcycled(gpu_lib):
    """Subcycled AMR with regrids: the source runs after every level update with
    that level's dt (merged launches read it per patch), before time interpolation."""
    cfg = cases.replace(cases.quadrants_amr(seed=1, minlevel=2, maxlevel=5, mx=8), src_term=1,
                        mthbc=(1, 1, 3, 1))
    o, d = _pair(cfg)
    t, dt = 0.0, cfg.initial_dt
    for k in range(4):
        c_o = o.advance(t, dt)
        assert d.advance_all_levels(t, dt) == c_o
        assert np.array_equal(d.get_q(), o.all_q()), f"macro step {k}"
        t += dt
        o.regrid()
        d.regrid()
        assert d.leaves() == o.leaves()
        assert np.array_equal(d.get_q(), o.all_q()), f"after regrid {k}"
        dt = dt * 0.9 / c_o


def test_src2_needs_the_euler_solver(gpu_lib):
    import forestclaw_b200 as fcb

    opts = cases.to_options(cases.replace(cases.radialdam_uniform(level=2, mx=16), src_term=1))
    with pytest.raises(fcb.FcbError) as e:
        fcb.Solver(opts)
    assert e.value.code == 1
