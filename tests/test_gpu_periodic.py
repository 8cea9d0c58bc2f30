"""Periodic domains and bricks on the CUDA path against the oracle.

A brick of b x b unmapped blocks (b a power of two; fclaw2d_map_brick.c maps
a patch of block (i, j) to ((i + xc)/b, (j + yc)/b)) is kept as one quadtree
whose levels count from the whole domain; periodic_x / periodic_y connect the
domain's opposite sides, so face and corner neighbours, 2:1 balance, smooth
refinement and every ghost-fill record (copies, averages, interpolations)
wrap around.  Every array bit for bit, through regrids.
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


def _steps(o, d, nmacro, dt, regrid=True):
    assert d.leaves() == o.leaves()
    assert np.array_equal(d.get_q(), o.all_q())
    t = 0.0
    for k in range(nmacro):
        c_o = o.advance(t, dt)
        assert d.advance_all_levels(t, dt) == c_o, k
        assert np.array_equal(d.get_q(), o.all_q()), f"macro step {k}"
        t += dt
        if regrid:
            o.regrid()
            d.regrid()
            assert d.leaves() == o.leaves(), f"mesh after regrid {k}"
            assert np.array_equal(d.get_q(), o.all_q()), f"after regrid {k}"
        dt = dt * 0.9 / c_o


def test_periodic_brick_advection_macro_steps(gpu_lib):
    """The periodic application's setup (2 x 2 brick, constant velocity (1, 1)
    in stored aux, disc initial data): the disc crosses the periodic corner."""
    cfg = cases.replace(O.periodic_regression(), pparams=(1.0, 1.0, 0.85, 0.85, 0.25))
    o, d = _pair(cfg)
    _steps(o, d, 5, cfg.initial_dt)


@pytest.mark.parametrize("claw_version", [4, 5])
def test_periodic_shallow_water_amr(gpu_lib, claw_version):
    """One periodic block (no brick), a dam break next to the periodic corner,
    levels 2-4 with subcycling and time interpolation."""
    cfg = cases.replace(cases.radialdam_amr(seed=0, minlevel=2, maxlevel=4, mx=16), periodic_x=1, periodic_y=1,
                        pparams=(0.9, 0.12, 0.2, 2.0, 1.0), claw_version=claw_version)
    o, d = _pair(cfg)
    if claw_version == 5:
        o_q = lambda: np.moveaxis(o.all_q(), 1, -1)  # noqa: E731
        assert d.leaves() == o.leaves()
        t, dt = 0.0, cfg.initial_dt
        for k in range(4):
            assert d.advance_all_levels(t, dt) == o.advance(t, dt)
            assert np.array_equal(d.get_q(), o_q()), k
            t += dt
            o.regrid()
            d.regrid()
            assert d.leaves() == o.leaves()
    else:
        _steps(o, d, 4, cfg.initial_dt)


def test_periodic_in_one_direction(gpu_lib):
    """periodic_x only: walls at the bottom and top, the left and right sides
    connected."""
    cfg = cases.replace(cases.radialdam_amr(seed=1, minlevel=2, maxlevel=4, mx=8), periodic_x=1,
                        mthbc=(1, 1, 3, 3), pparams=(0.05, 0.5, 0.2, 2.0, 1.0))
    o, d = _pair(cfg)
    _steps(o, d, 4, cfg.initial_dt)


@pytest.mark.parametrize("fusion", [1, 2])
def test_periodic_uniform_fused(gpu_lib, fusion):
    """A uniform periodic mesh: the fused step reads ghost cells across the
    periodic sides from the neighbours on the opposite side."""
    cfg = cases.replace(cases.radialdam_uniform(level=3, mx=16), periodic_x=1, periodic_y=1,
                        pparams=(0.1, 0.9, 0.2, 2.0, 1.0))
    o, d = _pair(cfg, ghost_fusion=fusion)
    _steps(o, d, 6, 0.4 / (16 * 8) / 1.5, regrid=False)
