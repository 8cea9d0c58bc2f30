"""Shared configurations: one Config (oracle) <-> Options (CUDA path) per case."""
from __future__ import annotations

import dataclasses

import numpy as np

import oracle as O


def to_options(cfg: O.Config):
    import forestclaw_b200 as fcb

    return fcb.Options(
        mx=cfg.mx, my=cfg.my, mbc=cfg.mbc, meqn=cfg.meqn, maux=cfg.maux,
        refinement_criteria=cfg.criteria, threshold_variable=cfg.ivar + 1,
        order=cfg.order, mcapa=cfg.mcapa, mwaves=cfg.mwaves, mthlim=cfg.mthlim, mthbc=cfg.mthbc,
        minlevel=cfg.minlevel, maxlevel=cfg.maxlevel, subcycle=cfg.subcycle,
        regrid_interval=cfg.regrid_interval, smooth_refine=cfg.smooth_refine,
        smooth_level=cfg.smooth_level, use_fixed_dt=cfg.use_fixed_dt, nout=cfg.nout,
        init_ghostcell=cfg.init_ghostcell, reduce_cfl=cfg.reduce_cfl,
        refine_threshold=cfg.refine_threshold, coarsen_threshold=cfg.coarsen_threshold,
        tfinal=cfg.tfinal, initial_dt=cfg.initial_dt, max_cfl=cfg.max_cfl,
        desired_cfl=cfg.desired_cfl, solver_kind=cfg.solver, problem=cfg.problem,
        grav=cfg.grav, gamma=cfg.gamma, problem_params=cfg.pparams, claw_version=cfg.claw_version,
        dry_tolerance=cfg.drytol, time_sync=cfg.time_sync, extent=cfg.extent, src_term=cfg.src_term,
        brick=cfg.brick, periodic_x=cfg.periodic_x, periodic_y=cfg.periodic_y,
    )


def swirl_uniform(level=4, mx=16, tperiod=2.0) -> O.Config:
    """Plain-method advection case: uniform level, MC limiter, order (2,2), swirl
    velocities with T = tperiod/2 (cos(pi t/T) at mid-step), q0 = 1 for x < 0.5."""
    return O.Config(mx=mx, my=mx, mbc=2, meqn=1, maux=2, order=(2, 2), mwaves=1, mthlim=(4,),
                    mthbc=(1, 1, 1, 1), minlevel=level, maxlevel=level, subcycle=1,
                    regrid_interval=0, use_fixed_dt=1, solver=O.ADVECTION, problem=O.SWIRL,
                    pparams=(tperiod,))


def swirl_dt(level=4, mx=16, cfl=0.9) -> float:
    """dt = cfl * dx / max|u| with max|u| = 1 on the unit square."""
    return cfl / (mx * (1 << level))


def radialdam_uniform(level=3, mx=16, r0=0.25, hin=2.0, hout=1.0) -> O.Config:
    return O.Config(mx=mx, my=mx, mbc=2, meqn=3, maux=0, order=(2, 2), mwaves=3, mthlim=(4, 4, 4),
                    mthbc=(1, 1, 1, 1), minlevel=level, maxlevel=level, regrid_interval=0,
                    use_fixed_dt=1, solver=O.SWE_ROE, problem=O.RADIALDAM, grav=1.0,
                    pparams=(0.5, 0.5, r0, hin, hout))


def quadrants_uniform(level=3, mx=16) -> O.Config:
    return O.Config(mx=mx, my=mx, mbc=2, meqn=4, maux=0, order=(2, 2), mwaves=4, mthlim=(4, 4, 4, 4),
                    mthbc=(1, 1, 1, 1), minlevel=level, maxlevel=level, regrid_interval=0,
                    use_fixed_dt=1, solver=O.EULER4_ROE, problem=O.QUADRANTS, gamma=1.4,
                    pparams=O.quadrants_params())


def radialdam_amr(seed=0, minlevel=3, maxlevel=6, mx=32, tfinal=0.5) -> O.Config:
    """AMR shallow water: Roe rpn2/rpt2, g = 1, subcycling, gradient tagging on h
    (refine > 0.05, coarsen < 0.01), regrid every step, smooth refinement,
    h = 2 inside r < r0 = 0.25 + 0.05*U(-1,1) (seeded), h = 1 outside."""
    rng = np.random.default_rng(seed)
    r0 = 0.25 + 0.05 * rng.uniform(-1.0, 1.0)
    return O.Config(mx=mx, my=mx, mbc=2, meqn=3, maux=0, order=(2, 2), mwaves=3, mthlim=(4, 4, 4),
                    mthbc=(1, 1, 1, 1), minlevel=minlevel, maxlevel=maxlevel, subcycle=1,
                    regrid_interval=1, smooth_refine=1, criteria=O.GRADIENT,
                    refine_threshold=0.05, coarsen_threshold=0.01, tfinal=tfinal,
                    initial_dt=0.9 / (mx * (1 << minlevel)) / 1.5, max_cfl=1.0, desired_cfl=0.9,
                    solver=O.SWE_ROE, problem=O.RADIALDAM, grav=1.0,
                    pparams=(0.5, 0.5, r0, 2.0, 1.0))


def quadrants_amr(seed=0, minlevel=2, maxlevel=7, mx=16, tfinal=0.25) -> O.Config:
    """AMR Euler (Roe with entropy fix, gamma = 1.4), subcycled: four quadrant
    states about (0.5, 0.5) drawn per seed, rho, p ~ U(0.1, 1.5) and
    u, v ~ U(-0.8, 0.8); gradient tagging on rho (refine > 1.0, coarsen < 0.1),
    regrid every step, adaptive dt."""
    rng = np.random.default_rng(seed)
    states = [(rng.uniform(0.1, 1.5), rng.uniform(-0.8, 0.8), rng.uniform(-0.8, 0.8), rng.uniform(0.1, 1.5))
              for _ in range(4)]
    return O.Config(mx=mx, my=mx, mbc=2, meqn=4, maux=0, order=(2, 2), mwaves=4, mthlim=(4, 4, 4, 4),
                    mthbc=(1, 1, 1, 1), minlevel=minlevel, maxlevel=maxlevel, subcycle=1,
                    regrid_interval=1, smooth_refine=1, criteria=O.GRADIENT,
                    refine_threshold=1.0, coarsen_threshold=0.1, tfinal=tfinal,
                    initial_dt=0.15 / (mx * (1 << minlevel)), max_cfl=1.0, desired_cfl=0.9,
                    solver=O.EULER4_ROE, problem=O.QUADRANTS, gamma=1.4,
                    pparams=O.quadrants_params(states, 0.5, 0.5))


def replace(cfg, **kw):
    return dataclasses.replace(cfg, **kw)


def bathy_lake(level=3, mx=16, seed=0, amp=1e-3, width=0.05, minlevel=None, maxlevel=None) -> O.Config:
    """Shallow water over a Gaussian bump, b = -1 + 0.8 exp(-r^2/0.02) about
    (0.5, 0.5): a lake at rest (eta = 0, h = -b >= 0.2) plus a surface pulse of
    amplitude `amp` and width `width` at a seeded place.  GeoClaw f-wave solver
    (rpn2_geoclaw + clawpack46_flux2fw), order (2, 0) since the reference's
    rpt2_geoclaw stops; g = 1, dry tolerance 1e-3, extrapolation boundaries."""
    rng = np.random.default_rng(seed)
    x0, y0 = rng.uniform(0.25, 0.75, size=2)
    lo = level if minlevel is None else minlevel
    hi = level if maxlevel is None else maxlevel
    return O.Config(mx=mx, my=mx, mbc=2, meqn=3, maux=1, order=(2, 0), mwaves=3, mthlim=(4, 4, 4),
                    mthbc=(1, 1, 1, 1), minlevel=lo, maxlevel=hi, subcycle=1,
                    regrid_interval=0 if lo == hi else 1, smooth_refine=1, criteria=O.GRADIENT,
                    refine_threshold=5e-3, coarsen_threshold=1e-3, use_fixed_dt=1,
                    solver=O.GEOCLAW_FWAVE, problem=O.BATHY, grav=1.0,
                    pparams=(float(x0), float(y0), amp, width))

