"""Option sets of the benchmarked workloads."""
from __future__ import annotations

from . import PROBLEM_SWIRL, SOLVER_ADVECTION, Options


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
