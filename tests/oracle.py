"""ctypes access to the CPU oracle (oracle/liboracle.so).

Test infrastructure only: the oracle is the checker for the CUDA path and is
never the thing measured or shipped.  The option arrays follow the layout
fixed in oracle/oracle_capi.cpp.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"

# Solver kinds (oracle/oracle_patch.hpp SolverKind)
ADVECTION, SWE_ROE, EULER4_ROE, GEOCLAW_FWAVE, ADVECTION_MANIFOLD = 0, 1, 2, 3, 4
# Problems (oracle/oracle_amr.hpp Problem)
SWIRL, RADIALDAM, QUADRANTS, BATHY, RADIALDAM_CELLAVE, HUMP, PERIODIC_DISC, FILAMENT = 0, 1, 2, 3, 4, 5, 6, 7
# Tagging criteria (oracle/oracle_clawpatch.hpp TagCriteria)
VALUE, MINMAX, DIFFERENCE, GRADIENT = 0, 1, 2, 3

_I_FIELDS = (["mx", "my", "mbc", "meqn", "maux", "order0", "order1", "mcapa", "mwaves"]
             + [f"mthlim{k}" for k in range(8)] + [f"mthbc{k}" for k in range(4)]
             + ["minlevel", "maxlevel", "subcycle", "regrid_interval", "smooth_refine",
                "smooth_level", "criteria", "ivar", "use_fixed_dt", "nout", "init_ghostcell",
                "reduce_cfl", "solver", "problem", "claw_version", "time_sync", "src_term", "brick",
                "periodic_x", "periodic_y"])
_D_FIELDS = (["refine_threshold", "coarsen_threshold", "tfinal", "initial_dt", "max_cfl",
              "desired_cfl", "grav", "gamma", "gamma1", "drytol"] + [f"p{k}" for k in range(32)]
             + ["ax", "bx", "ay", "by"])


@dataclass
class Config:
    """Options of one solve (names follow the reference's ini sections)."""
    mx: int = 16
    my: int = 16
    mbc: int = 2
    meqn: int = 1
    maux: int = 2
    order: tuple = (2, 2)
    mcapa: int = 0
    mwaves: int = 1
    mthlim: tuple = (4,)
    mthbc: tuple = (1, 1, 1, 1)
    minlevel: int = 4
    maxlevel: int = 4
    subcycle: int = 1
    regrid_interval: int = 1
    smooth_refine: int = 0
    smooth_level: int = 0
    criteria: int = MINMAX
    ivar: int = 0
    use_fixed_dt: int = 0
    nout: int = 1
    init_ghostcell: int = 0
    reduce_cfl: int = 1
    solver: int = ADVECTION
    problem: int = SWIRL
    refine_threshold: float = 0.5
    coarsen_threshold: float = 0.1
    tfinal: float = 1.0
    initial_dt: float = 0.01
    max_cfl: float = 1.0
    desired_cfl: float = 0.9
    grav: float = 1.0
    gamma: float = 1.4
    pparams: tuple = field(default_factory=tuple)
    claw_version: int = 4   # 4: fc2d_clawpack46, 5: fc2d_clawpack5
    drytol: float = 1e-3    # GeoClaw dry tolerance
    time_sync: int = 0      # [Options] time-sync: conservative coarse/fine correction
    extent: tuple = (0.0, 1.0, 0.0, 1.0)  # [Options] ax, bx, ay, by
    src_term: int = 0       # [clawpack46] src_term: 1 = the axisymmetric Euler source (shockbubble src2)
    brick: int = 1          # [Options] mi = mj: a brick of brick x brick blocks (a power of two)
    periodic_x: int = 0     # [Options] periodic_x
    periodic_y: int = 0     # [Options] periodic_y

    @property
    def gamma1(self) -> float:
        return self.gamma - 1.0

    def arrays(self):
        iv = {
            "mx": self.mx, "my": self.my, "mbc": self.mbc, "meqn": self.meqn, "maux": self.maux,
            "order0": self.order[0], "order1": self.order[1], "mcapa": self.mcapa,
            "mwaves": self.mwaves, "minlevel": self.minlevel, "maxlevel": self.maxlevel,
            "subcycle": self.subcycle, "regrid_interval": self.regrid_interval,
            "smooth_refine": self.smooth_refine, "smooth_level": self.smooth_level,
            "criteria": self.criteria, "ivar": self.ivar, "use_fixed_dt": self.use_fixed_dt,
            "nout": self.nout, "init_ghostcell": self.init_ghostcell,
            "reduce_cfl": self.reduce_cfl, "solver": self.solver, "problem": self.problem,
            "claw_version": self.claw_version, "time_sync": self.time_sync, "src_term": self.src_term,
            "brick": self.brick, "periodic_x": self.periodic_x, "periodic_y": self.periodic_y,
        }
        for k in range(8):
            iv[f"mthlim{k}"] = self.mthlim[k] if k < len(self.mthlim) else 0
        for k in range(4):
            iv[f"mthbc{k}"] = self.mthbc[k]
        dv = {
            "refine_threshold": self.refine_threshold, "coarsen_threshold": self.coarsen_threshold,
            "tfinal": self.tfinal, "initial_dt": self.initial_dt, "max_cfl": self.max_cfl,
            "desired_cfl": self.desired_cfl, "grav": self.grav, "gamma": self.gamma,
            "gamma1": self.gamma1, "drytol": self.drytol,
            "ax": self.extent[0], "bx": self.extent[1], "ay": self.extent[2], "by": self.extent[3],
        }
        for k in range(32):
            dv[f"p{k}"] = float(self.pparams[k]) if k < len(self.pparams) else 0.0
        ia = (ctypes.c_int * len(_I_FIELDS))(*[int(iv[n]) for n in _I_FIELDS])
        da = (ctypes.c_double * len(_D_FIELDS))(*[float(dv[n]) for n in _D_FIELDS])
        return ia, da

    @property
    def nx(self) -> int:
        return self.mx + 2 * self.mbc

    @property
    def ny(self) -> int:
        return self.my + 2 * self.mbc


_libs = {}
_lib_path = None


def use_library(path):
    """Select another build of the oracle (e.g. the OpenMP timing build) before first use."""
    global _lib_path
    _lib_path = Path(path)
    _libs.pop("plain", None)


def _build(target: str) -> Path:
    so = ORACLE_DIR / target
    srcs = list(ORACLE_DIR.glob("*.cpp")) + list(ORACLE_DIR.glob("*.hpp")) + [ORACLE_DIR / "Makefile"]
    if not so.exists() or any(s.stat().st_mtime > so.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", target], cwd=ORACLE_DIR, check=True)
    return so


def lib(parallel: bool = False):
    """Load (building on first use if needed) the oracle shared library.

    parallel: the OpenMP build of the same arithmetic (liboracle_omp.so: same
    compiler flags, the patches of a level updated by several threads), for
    the checks at full configuration sizes; its results equal the plain
    build's bit for bit."""
    key = "omp" if parallel else "plain"
    if key in _libs:
        return _libs[key]
    if parallel:
        so = _build("liboracle_omp.so")
    elif _lib_path is not None:
        so = _lib_path
    else:
        so = _build("liboracle.so")
    L = ctypes.CDLL(str(so))
    assert L.orc_iopt_count() == len(_I_FIELDS), "oracle option layout changed"
    assert L.orc_dopt_count() == len(_D_FIELDS), "oracle option layout changed"
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    L.orc_last_error.restype = ctypes.c_char_p
    L.orc_solver_new.restype = ctypes.c_void_p
    L.orc_solver_new.argtypes = [ip, dp]
    for name in ["orc_solver_free", "orc_initialize", "orc_run", "orc_regrid", "orc_num_patches"]:
        getattr(L, name).argtypes = [ctypes.c_void_p]
    L.orc_advance.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, dp]
    L.orc_update_single_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double, dp]
    L.orc_timeinterp_level.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
    L.orc_ghost_update.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int]
    L.orc_patch_info.argtypes = [ctypes.c_void_p, ctypes.c_int, ip, ip, ip]
    L.orc_get_q.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
    L.orc_set_q.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
    L.orc_get_qinterp.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
    L.orc_counters.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]
    L.orc_conservation.argtypes = [ctypes.c_void_p, dp]
    L.orc_neighbors.argtypes = [ctypes.c_void_p, ctypes.c_int, ip]
    L.orc_step2.argtypes = [ip, dp, dp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double, dp]
    L.orc_src2_axisymmetric.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 4 + [dp]
    _libs[key] = L
    return L


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(rc: int, L=None):
    if rc != 0:
        raise RuntimeError((L or lib()).orc_last_error().decode())


class OracleSolver:
    """One CPU solve: forest + patch data + counters.  parallel=True runs the
    OpenMP build of the same arithmetic (see lib())."""

    def __init__(self, cfg: Config, parallel: bool = False):
        self.cfg = cfg
        self._L = lib(parallel)
        ia, da = cfg.arrays()
        self._h = self._L.orc_solver_new(ia, da)
        if not self._h:
            raise RuntimeError(self._L.orc_last_error().decode())

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.orc_solver_free(self._h)
            self._h = None

    def initialize(self):
        _check(self._L.orc_initialize(self._h), self._L)

    def run(self):
        _check(self._L.orc_run(self._h))

    def advance(self, t: float, dt: float) -> float:
        c = ctypes.c_double()
        _check(self._L.orc_advance(self._h, t, dt, ctypes.byref(c)))
        return c.value

    def update_single_step(self, level: int, t: float, dt: float) -> float:
        c = ctypes.c_double()
        _check(self._L.orc_update_single_step(self._h, level, t, dt, ctypes.byref(c)))
        return c.value

    def timeinterp(self, level: int, alpha: float):
        _check(self._L.orc_timeinterp_level(self._h, level, alpha))

    def ghost_update(self, minlevel: int, maxlevel: int, t: float = 0.0, time_interp: int = 0):
        _check(self._L.orc_ghost_update(self._h, minlevel, maxlevel, t, time_interp))

    def regrid(self):
        _check(self._L.orc_regrid(self._h))

    @property
    def num_patches(self) -> int:
        return self._L.orc_num_patches(self._h)

    def patch_info(self, p: int):
        lv, x, y = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._L.orc_patch_info(self._h, p, ctypes.byref(lv), ctypes.byref(x), ctypes.byref(y))
        return lv.value, x.value, y.value

    def leaves(self):
        return [self.patch_info(p) for p in range(self.num_patches)]

    def q(self, p: int) -> np.ndarray:
        c = self.cfg
        out = np.empty((c.meqn, c.ny, c.nx), dtype=np.float64)
        self._L.orc_get_q(self._h, p, _dptr(out))
        return out

    def qinterp(self, p: int) -> np.ndarray:
        c = self.cfg
        out = np.empty((c.meqn, c.ny, c.nx), dtype=np.float64)
        self._L.orc_get_qinterp(self._h, p, _dptr(out))
        return out

    def all_q(self) -> np.ndarray:
        return np.stack([self.q(p) for p in range(self.num_patches)])

    def set_q(self, p: int, q: np.ndarray):
        a = np.ascontiguousarray(q, dtype=np.float64)
        self._L.orc_set_q(self._h, p, _dptr(a))

    def counters(self):
        a = (ctypes.c_longlong * 4)()
        self._L.orc_counters(self._h, a)
        return {"count_amr_advance": a[0], "count_amr_new_domain": a[1],
                "count_amr_regrid": a[2], "count_single_step": a[3]}

    def conservation(self) -> np.ndarray:
        out = np.zeros(self.cfg.meqn)
        self._L.orc_conservation(self._h, _dptr(out))
        return out

    def neighbors(self, p: int):
        a = (ctypes.c_int * 22)()
        self._L.orc_neighbors(self._h, p, a)
        return list(a)


def step2(cfg: Config, q: np.ndarray, aux, dx: float, dy: float, dt: float) -> float:
    """One clawpack46 patch update in place; returns the patch CFL number."""
    ia, da = cfg.arrays()
    c = ctypes.c_double()
    auxp = _dptr(aux) if aux is not None else ctypes.POINTER(ctypes.c_double)()
    _check(lib().orc_step2(ia, da, _dptr(q), auxp, dx, dy, dt, ctypes.byref(c)))
    return c.value


def src2_axisymmetric(q: np.ndarray, mbc: int, ylower: float, dy: float, gamma1: float, dt: float):
    """The oracle's src2 (euler/2d/shockbubble/user_4.6/src2.f) on one patch
    q[m, j, i] in place."""
    meqn, ny, nx = q.shape
    a = np.ascontiguousarray(q)
    _check(lib().orc_src2_axisymmetric(nx - 2 * mbc, ny - 2 * mbc, mbc, meqn, ylower, dy, gamma1, dt, _dptr(a)))
    q[...] = a


# ---- configurations of the reference regression tests -----------------------
def swirl_regression(claw_version: int = 4) -> Config:
    """applications/clawpack/advection/2d/swirl/regression.ini"""
    return Config(mx=8, my=8, mbc=2, meqn=1, maux=3, order=(2, 2), mwaves=1, mthlim=(3,),
                  mthbc=(1, 1, 1, 1), minlevel=2, maxlevel=6, regrid_interval=1,
                  refine_threshold=0.25, coarsen_threshold=0.05, smooth_refine=1,
                  tfinal=0.1, initial_dt=0.005, max_cfl=1.0, desired_cfl=0.9, nout=1,
                  subcycle=1, solver=ADVECTION, problem=SWIRL, criteria=MINMAX,
                  pparams=(4.0,), claw_version=claw_version)


def radialdam_regression(claw_version: int = 4) -> Config:
    """applications/clawpack/shallow/2d/radialdam/regression.ini on top of that
    directory's fclaw_options.ini (read first, fclaw_base.c:758-786), which sets
    refinement-criteria = gradient; example 0: unmapped [-2.5, 2.5]^2, cellave2
    initial depth, shallow-water Roe solver with time-sync = T."""
    return Config(mx=16, my=16, mbc=2, meqn=3, maux=0, order=(2, 2), mwaves=3, mthlim=(4, 4, 4),
                  mthbc=(1, 1, 1, 1), minlevel=1, maxlevel=5, regrid_interval=1,
                  refine_threshold=0.5, coarsen_threshold=0.25, smooth_refine=1, smooth_level=4,
                  tfinal=0.4, initial_dt=0.0625, max_cfl=1.0, desired_cfl=0.9, nout=1,
                  subcycle=1, solver=SWE_ROE, problem=RADIALDAM_CELLAVE, criteria=GRADIENT, grav=1.0,
                  pparams=(0.0, 0.0, 0.5, 2.0, 1.0), claw_version=claw_version, time_sync=1,
                  extent=(-2.5, 2.5, -2.5, 2.5))


def bump_regression(claw_version: int = 4) -> Config:
    """applications/clawpack/shallow/2d/bump/regression.ini on top of that
    directory's fclaw_options.ini (read first), which sets refinement-criteria =
    minmax: unmapped [-2.5, 2.5]^2, mx = 8, levels 4-6, smooth-level 4,
    h = 0.1 + exp(-200 r^2) about the origin (user_4.6/qinit.f), shallow-water
    Roe solver, g = 1.  The clawpack 4.6 run has extrapolation boundaries
    ([clawpack46] mthbc = 1 1 1 1), the clawpack 5 run solid walls
    ([clawpack5] mthbc = 3 3 3 3)."""
    return Config(mx=8, my=8, mbc=2, meqn=3, maux=0, order=(2, 2), mwaves=3, mthlim=(4, 4, 4),
                  mthbc=(1, 1, 1, 1) if claw_version == 4 else (3, 3, 3, 3), minlevel=4, maxlevel=6,
                  regrid_interval=1, refine_threshold=0.05, coarsen_threshold=0.005, smooth_refine=1,
                  smooth_level=4, tfinal=1.0, initial_dt=2.5e-2, max_cfl=1.0, desired_cfl=0.9, nout=1,
                  subcycle=1, solver=SWE_ROE, problem=HUMP, criteria=MINMAX, grav=1.0,
                  pparams=(0.0, 0.0, 0.1, 200.0), claw_version=claw_version,
                  extent=(-2.5, 2.5, -2.5, 2.5))


def periodic_regression(claw_version: int = 4) -> Config:
    """applications/clawpack/advection/2d/periodic/regression.ini on top of
    that directory's fclaw_options.ini (minmax tagging): a 2 x 2 brick on
    [-1, 1]^2, periodic in x and y, mx = 8, levels 2-5 of each block, constant
    velocity (1, 1) in aux(1:2) (maux = 3), q = the fraction of each cell inside
    the disc of radius 0.25 about the origin; rpn2adv/rpt2adv with the van Leer
    limiter (mthlim = 3); smooth-level = 5 from fclaw_options.ini."""
    return Config(mx=8, my=8, mbc=2, meqn=1, maux=3, order=(2, 2), mwaves=1, mthlim=(3,),
                  mthbc=(1, 1, 1, 1), minlevel=2, maxlevel=5, regrid_interval=1,
                  refine_threshold=0.25, coarsen_threshold=0.05, smooth_refine=1, smooth_level=5,
                  tfinal=0.2, initial_dt=0.02, max_cfl=1.0, desired_cfl=0.9, nout=1,
                  subcycle=1, solver=ADVECTION, problem=PERIODIC_DISC, criteria=MINMAX,
                  pparams=(1.0, 1.0, 0.0, 0.0, 0.25), claw_version=claw_version,
                  extent=(-1.0, 1.0, -1.0, 1.0), brick=2, periodic_x=1, periodic_y=1)


def filament_regression(claw_version: int = 4) -> Config:
    """applications/clawpack/advection/2d/filament/regression_map.ini with
    --user:example=1 on top of that directory's fclaw_options.ini (minmax
    tagging): a 2 x 2 brick under the cart mapping shifted by (1, 1), i.e.
    [0, 2]^2, manifold = T, capacity aux(1) (mcapa = 1), edge velocities from
    psi = (4/3) r^3 about (1, 1) in aux(2:3) (user46_setaux_manifold.f), the
    manifold advection solvers, q = the fraction of each cell inside the disc of
    radius 0.25 about (0.5, 1) (fdisc.f, cellave2.f), mx = 16, levels 3-5 of
    each block, van Leer limiter, t = 0 .. 0.025 from dt = 0.0025."""
    return Config(mx=16, my=16, mbc=2, meqn=1, maux=3, order=(2, 2), mcapa=1, mwaves=1, mthlim=(3,),
                  mthbc=(1, 1, 1, 1), minlevel=3, maxlevel=5, regrid_interval=1,
                  refine_threshold=0.25, coarsen_threshold=0.05, smooth_refine=1, smooth_level=5,
                  tfinal=0.025, initial_dt=0.0025, max_cfl=1.0, desired_cfl=0.9, nout=1,
                  subcycle=1, solver=ADVECTION_MANIFOLD, problem=FILAMENT, criteria=MINMAX,
                  pparams=(0.0, 0.0, 0.5, 1.0, 0.25), claw_version=claw_version,
                  extent=(0.0, 2.0, 0.0, 2.0), brick=2)


QUADRANT_STATES = (
    # rho, u, v, p for quadrants 1..4 (euler/2d/quadrants/user_4.6/qinit.f)
    (1.5, 0.0, 0.0, 1.5),
    (0.532258064516129, 1.206045378311055, 0.0, 0.3),
    (0.137992831541219, 1.206045378311055, 1.206045378311055, 0.029032258064516),
    (0.532258064516129, 0.0, 1.206045378311055, 0.3),
)


def quadrants_params(states=QUADRANT_STATES, xs=0.8, ys=0.8):
    rho = [s[0] for s in states]
    u = [s[1] for s in states]
    v = [s[2] for s in states]
    p = [s[3] for s in states]
    return tuple(rho + u + v + p + [xs, ys])


def quadrants_regression(claw_version: int = 4) -> Config:
    """applications/clawpack/euler/2d/quadrants/regression.ini on top of that directory's
    fclaw_options.ini, which the application reads first from its working directory
    (fclaw_base.c:758-786); that file sets refinement-criteria = difference.  The
    [clawpack46] and [clawpack5] sections agree (extrapolation boundaries)."""
    return Config(mx=8, my=8, mbc=2, meqn=4, maux=0, order=(2, 2), mwaves=4, mthlim=(4, 4, 4, 4),
                  mthbc=(1, 1, 1, 1), minlevel=0, maxlevel=5, regrid_interval=1,
                  refine_threshold=0.25, coarsen_threshold=0.025, smooth_refine=1, smooth_level=5,
                  tfinal=0.1, initial_dt=0.05, max_cfl=1.0, desired_cfl=0.9, nout=1,
                  subcycle=1, solver=EULER4_ROE, problem=QUADRANTS, criteria=DIFFERENCE, gamma=1.4,
                  pparams=quadrants_params(), claw_version=claw_version)
