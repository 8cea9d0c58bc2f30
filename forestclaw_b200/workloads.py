"""Option sets of the benchmarked workloads (synthetic, seeded inputs)."""
from __future__ import annotations

import numpy as np

from . import (PROBLEM_BATHY, PROBLEM_FILAMENT, PROBLEM_QUADRANTS, PROBLEM_RADIALDAM, PROBLEM_SWIRL,
               SOLVER_ADVECTION, SOLVER_ADVECTION_MANIFOLD, SOLVER_EULER4_ROE, SOLVER_GEOCLAW_FWAVE, SOLVER_SWE_ROE,
               TAG_GRADIENT, TAG_MINMAX, Options)


def uniform_swirl(level: int = 8, mx: int = 16) -> Options:
    """Uniform swirl advection (advection/2d/swirl with the plain method): meqn = 1,
    MC limiter, order (2,2), extrapolation boundaries, velocities
    u = sin^2(pi x) sin(2 pi y) cos(pi t), v = -sin^2(pi y) sin(2 pi x) cos(pi t)
    (the reference's stream-function differences with tperiod = 2), q0 = 1 for x < 0.5."""
    return Options(mx=mx, my=mx, mbc=2, meqn=1, maux=2, order=(2, 2), mwaves=1, mthlim=(4,),
                   mthbc=(1, 1, 1, 1), minlevel=level, maxlevel=level, subcycle=1, regrid_interval=0,
                   use_fixed_dt=1, solver_kind=SOLVER_ADVECTION, problem=PROBLEM_SWIRL,
                   problem_params=(2.0,))


def swirl_dt(level: int = 8, mx: int = 16, cfl: float = 0.9) -> float:
    """dt = cfl * dx / max|u| with max|u| = 1."""
    return cfl / (mx * (1 << level))


def amr_shallow_water(seed: int = 0, minlevel: int = 3, maxlevel: int = 6, mx: int = 32,
                      tfinal: float = 0.5) -> Options:
    """AMR shallow water: Roe rpn2/rpt2 with entropy fix, g = 1, unit square,
    subcycling, gradient tagging on h (refine > 0.05, coarsen < 0.01), regrid
    every step, smooth refinement; dam break h = 2 inside r < r0 = 0.25 +
    0.05*U(-1,1) (one seeded draw) about (0.5, 0.5), h = 1 outside, at rest."""
    rng = np.random.default_rng(seed)
    r0 = 0.25 + 0.05 * rng.uniform(-1.0, 1.0)
    return Options(mx=mx, my=mx, mbc=2, meqn=3, maux=0, order=(2, 2), mwaves=3, mthlim=(4, 4, 4),
                   mthbc=(1, 1, 1, 1), minlevel=minlevel, maxlevel=maxlevel, subcycle=1, regrid_interval=1,
                   smooth_refine=1, refinement_criteria=TAG_GRADIENT, refine_threshold=0.05,
                   coarsen_threshold=0.01, tfinal=tfinal, initial_dt=0.9 / (mx * (1 << minlevel)) / 1.5,
                   max_cfl=1.0, desired_cfl=0.9, solver_kind=SOLVER_SWE_ROE, problem=PROBLEM_RADIALDAM,
                   grav=1.0, problem_params=(0.5, 0.5, float(r0), 2.0, 1.0))


def amr_euler(seed: int = 0, minlevel: int = 2, maxlevel: int = 7, mx: int = 16, tfinal: float = 0.25) -> Options:
    """AMR Euler (Roe with entropy fix, gamma = 1.4), subcycled: four quadrant
    states about (0.5, 0.5) drawn per seed, rho, p ~ U(0.1, 1.5) and
    u, v ~ U(-0.8, 0.8); gradient tagging on rho (refine > 1.0, coarsen < 0.1),
    regrid every step, adaptive dt."""
    rng = np.random.default_rng(seed)
    states = [(rng.uniform(0.1, 1.5), rng.uniform(-0.8, 0.8), rng.uniform(-0.8, 0.8), rng.uniform(0.1, 1.5))
              for _ in range(4)]
    params = ([s[0] for s in states] + [s[1] for s in states] + [s[2] for s in states] + [s[3] for s in states]
              + [0.5, 0.5])
    return Options(mx=mx, my=mx, mbc=2, meqn=4, maux=0, order=(2, 2), mwaves=4, mthlim=(4, 4, 4, 4),
                   mthbc=(1, 1, 1, 1), minlevel=minlevel, maxlevel=maxlevel, subcycle=1, regrid_interval=1,
                   smooth_refine=1, refinement_criteria=TAG_GRADIENT, refine_threshold=1.0, coarsen_threshold=0.1,
                   tfinal=tfinal, initial_dt=0.15 / (mx * (1 << minlevel)), max_cfl=1.0, desired_cfl=0.9,
                   solver_kind=SOLVER_EULER4_ROE, problem=PROBLEM_QUADRANTS, gamma=1.4,
                   problem_params=tuple(float(v) for v in params))


def bathymetry(seed: int = 0, minlevel: int = 4, maxlevel: int = 7, mx: int = 32, amp: float = 1e-3,
               width: float = 0.05) -> Options:
    """Shallow water over b = -1 + 0.8 exp(-((x-.5)^2+(y-.5)^2)/0.02): a lake at
    rest (eta = 0) plus a surface pulse of amplitude `amp` and width `width` at
    a seeded place; GeoClaw f-wave solver, order (2, 0), g = 1, dry tolerance
    1e-3, subcycled, gradient tagging, regrid every step, fixed dt."""
    rng = np.random.default_rng(seed)
    x0, y0 = rng.uniform(0.25, 0.75, size=2)
    return Options(mx=mx, my=mx, mbc=2, meqn=3, maux=1, order=(2, 0), mwaves=3, mthlim=(4, 4, 4),
                   mthbc=(1, 1, 1, 1), minlevel=minlevel, maxlevel=maxlevel, subcycle=1,
                   regrid_interval=0 if minlevel == maxlevel else 1, smooth_refine=1,
                   refinement_criteria=TAG_GRADIENT, refine_threshold=5e-3, coarsen_threshold=1e-3, use_fixed_dt=1,
                   solver_kind=SOLVER_GEOCLAW_FWAVE, problem=PROBLEM_BATHY, grav=1.0,
                   problem_params=(float(x0), float(y0), amp, width))


def bathymetry_dt(minlevel: int = 4, mx: int = 32) -> float:
    """CFL about 0.5 on the coarsest level (|u| + sqrt(g h) <= 1)."""
    return 0.5 / (mx * (1 << minlevel))


def dam_break_requests(n: int, seed: int, maxlevels=(4, 5, 6, 7), tfinal=(0.2, 1.0), mxs=(16, 32),
                       subcycle: int = 1):
    """Ensemble-serving requests: dam breaks about (0.5, 0.5) with radius
    ~ U(0.1, 0.3), inner depth ~ U(1.5, 3), outer depth 1, maxlevel uniform
    over `maxlevels`, mx uniform over `mxs`, final time ~ U(tfinal); levels
    from 2, subcycled (the reference's default) unless subcycle = 0, regrid
    every macro step, adaptive dt (desired CFL 0.9)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        r0, hin = rng.uniform(0.1, 0.3), rng.uniform(1.5, 3.0)
        maxlevel = int(rng.choice(list(maxlevels)))
        mx = int(rng.choice(list(mxs)))
        tf = float(rng.uniform(*tfinal))
        o = amr_shallow_water(seed=0, minlevel=2, maxlevel=maxlevel, mx=mx, tfinal=tf)
        o.problem_params = (0.5, 0.5, float(r0), float(hin), 1.0)
        o.initial_dt = 0.9 / (mx * 4) / (hin ** 0.5 + 1)
        o.subcycle = subcycle
        out.append(o)
    return out


def filament(minlevel: int = 4, maxlevel: int = 6, mx: int = 32, claw_version: int = 4) -> Options:
    """The filament application (advection/2d/filament, example 1) on a finer
    mesh: a 2 x 2 brick under the cart mapping, [0, 2]^2, capacity in aux(1)
    (mcapa = 1) and the edge velocities of psi = (4/3) r^3 about (1, 1) in
    aux(2:3), manifold advection solvers, van Leer limiter, minmax tagging
    (refine > 0.25, coarsen < 0.05), the disc of radius 0.25 about (0.5, 1) as
    cell fractions; levels per block, subcycled, regrid every step, adaptive dt
    (initial dt: CFL 0.9 at the largest edge speed, 8, on the coarsest level)."""
    return Options(mx=mx, my=mx, mbc=2, meqn=1, maux=3, order=(2, 2), mcapa=1, mwaves=1, mthlim=(3,),
                   mthbc=(1, 1, 1, 1), minlevel=minlevel, maxlevel=maxlevel, subcycle=1, regrid_interval=1,
                   smooth_refine=1, smooth_level=maxlevel, refinement_criteria=TAG_MINMAX, refine_threshold=0.25,
                   coarsen_threshold=0.05, tfinal=0.1, initial_dt=0.9 / (8.0 * mx * (1 << minlevel)),
                   max_cfl=1.0, desired_cfl=0.9, solver_kind=SOLVER_ADVECTION_MANIFOLD, problem=PROBLEM_FILAMENT,
                   problem_params=(0.0, 0.0, 0.5, 1.0, 0.25), claw_version=claw_version,
                   extent=(0.0, 2.0, 0.0, 2.0), brick=2)
