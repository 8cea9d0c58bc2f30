"""Mapped grids with capacity on the CUDA path against the oracle.

The filament application (applications/clawpack/advection/2d/filament,
example 1): a 2 x 2 brick under the cart mapping with manifold = T, the
capacity kappa = area/(dx dy) in aux(1) (mcapa = 1) and the edge velocities of
psi = (4/3) r^3 in aux(2:3), advanced by clawpack46_rpn2adv_manifold /
rpt2adv_manifold with the capacity form of the step: dtdx1d(i) = dtdx/kappa(i)
in the CFL number, the limiter's dtdxave and the transverse splits
(clawpack46_step2.f:122-126,191-195, clawpack46_flux2.f:134-220), and
q -= (dtdx*df + dtdy*dg)/kappa (clawpack46_step2_wrap.f:118-121).

On this mesh the mapped corners are dyadic, so kappa is exactly 1; the tests
that set p[0] multiply it by 1 + p[0]*xc*yc so that dtdx1d differs from cell to
cell and every choice of dtdx1d(i-1) or dtdx1d(i) shows in the bits.
"""
import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu


def _pair(cfg):
    import forestclaw_b200 as fcb

    o = O.OracleSolver(cfg)
    d = fcb.Solver(cases.to_options(cfg))
    o.initialize()
    d.initialize()
    return o, d


def _oq(o):
    """Oracle arrays in fcb_get_q's order: (patch, m, j, i), or (patch, j, i, m) for clawpack 5."""
    q = o.all_q()
    return np.moveaxis(q, 1, -1) if o.cfg.claw_version == 5 else q


def _macro_steps(o, d, nmacro, dt, regrid=True):
    assert d.leaves() == o.leaves()
    assert np.array_equal(d.get_q(), _oq(o))
    t = 0.0
    for k in range(nmacro):
        c_o = o.advance(t, dt)
        assert d.advance_all_levels(t, dt) == c_o, k
        assert np.array_equal(d.get_q(), _oq(o)), f"macro step {k}"
        t += dt
        if regrid:
            o.regrid()
            d.regrid()
            assert d.leaves() == o.leaves(), f"mesh after regrid {k}"
            assert np.array_equal(d.get_q(), _oq(o)), f"after regrid {k}"
        dt = dt * 0.9 / c_o


@pytest.mark.parametrize("claw_version", [4, 5])
@pytest.mark.parametrize("kmod", [0.0, 0.4])
def test_filament_amr_macro_steps(gpu_lib, kmod, claw_version):
    """Levels 3-5 of each block with subcycling, time interpolation and a regrid
    after every macro step, bit for bit (kmod = 0: the application's setup);
    clawpack 5 updates the interior cells only (clawpack5_step2_wrap.f)."""
    cfg = cases.replace(O.filament_regression(claw_version), pparams=(kmod, 0.0, 0.5, 1.0, 0.25))
    o, d = _pair(cfg)
    _macro_steps(o, d, 6, cfg.initial_dt)


@pytest.mark.parametrize("claw_version", [4, 5])
@pytest.mark.parametrize("mx", [8, 16, 32, 64])
def test_filament_uniform_capacity(gpu_lib, mx, claw_version):
    """One level of the brick with a varying capacity: every patch size of the
    four-barrier form, CFL numbers and fields bit for bit."""
    cfg = cases.replace(O.filament_regression(claw_version), mx=mx, my=mx, minlevel=2, maxlevel=2,
                        pparams=(0.7, 0.0, 0.5, 1.0, 0.25))
    o, d = _pair(cfg)
    _macro_steps(o, d, 4, 0.5 * cfg.initial_dt * 16 / mx, regrid=False)


def test_filament_served_equals_run(gpu_lib):
    """A filament solve through the serving loop, mixed with a shallow-water
    solve, ends with the same field as fcb_run (the batched launch of the
    four-barrier form reads each patch's capacity through its descriptor)."""
    import forestclaw_b200 as fcb
    from forestclaw_b200.serve import Server

    cfg = cases.replace(O.filament_regression(4), pparams=(0.4, 0.0, 0.5, 1.0, 0.25))
    alone = fcb.Solver(cases.to_options(cfg))
    alone.initialize()
    alone.run()
    other = cases.radialdam_amr(seed=1, minlevel=2, maxlevel=4, mx=16, tfinal=0.05)
    srv = Server(1 << 40)
    try:
        ids = [srv.submit(cases.to_options(cfg)), srv.submit(cases.to_options(other))]
        srv.run_until_idle()
        q = srv.get_q(ids[0])
    finally:
        srv.close()
    assert np.array_equal(q, alone.get_q())
