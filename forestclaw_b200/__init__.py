"""forestclaw_b200: the ForestClaw patch hot path on NVIDIA B200 (sm_100a).

Python binding of the C ABI in include/fclaw_b200.h.  The names follow the
reference's time-stepping core (fclaw2d_initialize, fclaw2d_run,
fclaw2d_advance_all_levels, fclaw2d_update_single_step, fclaw2d_ghost_update,
fclaw2d_timeinterp, fclaw2d_regrid) and its option sections ([clawpatch],
[clawpack46], [Options]).

The CUDA library is required: loading fails loudly if libfclaw_b200.so is
missing, and there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

__all__ = ["Options", "Solver", "Comm", "local_group", "nccl_unique_id", "nccl_comm", "partition_plan", "lib",
           "FcbError", "SOLVER_ADVECTION", "SOLVER_SWE_ROE",
           "SOLVER_EULER4_ROE", "SOLVER_GEOCLAW_FWAVE", "SOLVER_ADVECTION_MANIFOLD", "PROBLEM_SWIRL",
           "PROBLEM_RADIALDAM", "PROBLEM_QUADRANTS", "PROBLEM_BATHY", "PROBLEM_RADIALDAM_CELLAVE", "PROBLEM_HUMP",
           "PROBLEM_PERIODIC_DISC", "PROBLEM_FILAMENT",
           "PRECISION_FP64", "PRECISION_MIXED", "measure_fp_rate",
           "TAG_VALUE", "TAG_MINMAX", "TAG_DIFFERENCE", "TAG_GRADIENT", "EXPORTED_SYMBOLS"]

PKG = Path(__file__).resolve().parent
LIBPATH = PKG / "libfclaw_b200.so"

SOLVER_ADVECTION, SOLVER_SWE_ROE, SOLVER_EULER4_ROE, SOLVER_GEOCLAW_FWAVE = 0, 1, 2, 3
SOLVER_ADVECTION_MANIFOLD = 4
PROBLEM_SWIRL, PROBLEM_RADIALDAM, PROBLEM_QUADRANTS, PROBLEM_BATHY, PROBLEM_RADIALDAM_CELLAVE = 0, 1, 2, 3, 4
PROBLEM_HUMP = 5
PROBLEM_PERIODIC_DISC = 6
PROBLEM_FILAMENT = 7
PRECISION_FP64, PRECISION_MIXED = 0, 1
TAG_VALUE, TAG_MINMAX, TAG_DIFFERENCE, TAG_GRADIENT = 0, 1, 2, 3

EXPORTED_SYMBOLS = (
    "fcb_abi_version", "fcb_advance_all_levels", "fcb_conservation_check", "fcb_context_create",
    "fcb_context_destroy", "fcb_counters", "fcb_curr_time", "fcb_get_q", "fcb_get_qinterp",
    "fcb_ghost_update", "fcb_initialize", "fcb_last_error", "fcb_num_patches", "fcb_patch_info",
    "fcb_patch_neighbors", "fcb_patch_size", "fcb_physical_set_bc", "fcb_regrid", "fcb_run",
    "fcb_set_q", "fcb_single_step_update", "fcb_synchronize", "fcb_timeinterp",
    "fcb_update_single_step", "fcb_update_single_step_async", "fcb_conservation_sum_noalloc",
    "fcb_server_create", "fcb_server_destroy", "fcb_server_submit", "fcb_server_round", "fcb_server_status",
    "fcb_server_get_q", "fcb_server_release", "fcb_server_clock", "fcb_autotune_info",
    "fcb_measure_fp_rate", "fcb_output_ascii", "fcb_comm_create_local", "fcb_comm_nccl_unique_id",
    "fcb_comm_create_nccl", "fcb_comm_destroy", "fcb_context_create_partitioned", "fcb_partition_info",
    "fcb_global_maximum", "fcb_partition_plan", "fcb_step_kernel_time", "fcb_server_set_work_limit",
    "fcb_advance_all_levels_async", "fcb_read_max_cfl",
)


class _Options(ctypes.Structure):
    """Mirror of fcb_options_t."""
    _fields_ = [
        ("mx", ctypes.c_int), ("my", ctypes.c_int), ("mbc", ctypes.c_int), ("meqn", ctypes.c_int),
        ("maux", ctypes.c_int), ("refinement_criteria", ctypes.c_int),
        ("threshold_variable", ctypes.c_int),
        ("order", ctypes.c_int * 2), ("mcapa", ctypes.c_int), ("mwaves", ctypes.c_int),
        ("mthlim", ctypes.c_int * 8), ("mthbc", ctypes.c_int * 4),
        ("minlevel", ctypes.c_int), ("maxlevel", ctypes.c_int), ("subcycle", ctypes.c_int),
        ("regrid_interval", ctypes.c_int), ("smooth_refine", ctypes.c_int),
        ("smooth_level", ctypes.c_int), ("use_fixed_dt", ctypes.c_int), ("nout", ctypes.c_int),
        ("init_ghostcell", ctypes.c_int), ("reduce_cfl", ctypes.c_int),
        ("refine_threshold", ctypes.c_double), ("coarsen_threshold", ctypes.c_double),
        ("tfinal", ctypes.c_double), ("initial_dt", ctypes.c_double), ("max_cfl", ctypes.c_double),
        ("desired_cfl", ctypes.c_double),
        ("solver_kind", ctypes.c_int), ("problem", ctypes.c_int),
        ("grav", ctypes.c_double), ("gamma", ctypes.c_double),
        ("problem_params", ctypes.c_double * 32),
        ("step_variant", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("macro_graph", ctypes.c_int),
        ("claw_version", ctypes.c_int),
        ("dry_tolerance", ctypes.c_double),
        ("time_sync", ctypes.c_int),
        ("ax", ctypes.c_double), ("bx", ctypes.c_double), ("ay", ctypes.c_double), ("by", ctypes.c_double),
        ("weighted_partition", ctypes.c_int),
        ("ghost_fusion", ctypes.c_int),
        ("src_term", ctypes.c_int),
        ("brick", ctypes.c_int), ("periodic_x", ctypes.c_int), ("periodic_y", ctypes.c_int),
    ]


class RequestStatus(ctypes.Structure):
    """Mirror of fcb_request_status_t."""
    _fields_ = [("state", ctypes.c_int), ("num_patches", ctypes.c_int), ("t", ctypes.c_double),
                ("submit_s", ctypes.c_double), ("start_s", ctypes.c_double), ("finish_s", ctypes.c_double),
                ("cell_updates", ctypes.c_longlong), ("count_amr_advance", ctypes.c_longlong)]


class _Counters(ctypes.Structure):
    _fields_ = [(n, ctypes.c_longlong) for n in (
        "count_amr_advance", "count_amr_new_domain", "count_amr_regrid", "count_single_step",
        "count_ghost_waves", "count_kernel_launches", "count_graph_replays")]


@dataclass
class Options:
    """Options of one solve, named as in the reference's ini sections."""
    # [clawpatch]
    mx: int = 16
    my: int = 16
    mbc: int = 2
    meqn: int = 1
    maux: int = 2
    refinement_criteria: int = TAG_MINMAX
    threshold_variable: int = 1
    # [clawpack46]
    order: Sequence[int] = (2, 2)
    mcapa: int = 0
    mwaves: int = 1
    mthlim: Sequence[int] = (4,)
    mthbc: Sequence[int] = (1, 1, 1, 1)
    # [Options]
    minlevel: int = 4
    maxlevel: int = 4
    subcycle: int = 1
    regrid_interval: int = 1
    smooth_refine: int = 0
    smooth_level: int = 0
    use_fixed_dt: int = 0
    nout: int = 1
    init_ghostcell: int = 0
    reduce_cfl: int = 1
    refine_threshold: float = 0.5
    coarsen_threshold: float = 0.1
    tfinal: float = 1.0
    initial_dt: float = 0.01
    max_cfl: float = 1.0
    desired_cfl: float = 0.9
    # solver / problem
    solver_kind: int = SOLVER_ADVECTION
    problem: int = PROBLEM_SWIRL
    grav: float = 1.0
    gamma: float = 1.4
    problem_params: Sequence[float] = field(default_factory=tuple)
    # step kernel form: 0 = library's choice, 1 = CTA rows, 2 = warp-synchronous, 3 = pipelined
    step_variant: int = 0
    # 0 = FP64 throughout, 1 = mixed FP32 solves / FP64 accumulation
    precision: int = PRECISION_FP64
    # 1: advance_all_levels replays the macro-step as one CUDA graph; 0: host
    # launches; 2: automatic (the graph whenever a macro step updates a level)
    macro_graph: int = 2
    # 4: fc2d_clawpack46 update, 5: fc2d_clawpack5 update (arrays in q(m,i,j) order)
    claw_version: int = 4
    # GeoClaw /common_swe/ dry_tolerance
    dry_tolerance: float = 1e-3
    # [Options] time-sync: conservative coarse/fine and same-size corrections
    time_sync: int = 0
    # [Options] ax, bx, ay, by: physical extent of the block
    extent: Sequence[float] = (0.0, 1.0, 0.0, 1.0)
    # [Options] weighted-partition: partitioned solves weigh leaves by 2^level when subcycling
    weighted_partition: int = 1
    # ghost-exchange fusion on a mesh of one level: 0 autotuned, 1 off, 2 on
    ghost_fusion: int = 0
    # [clawpack46] src_term: 1 = the axisymmetric Euler source (shockbubble src2)
    src_term: int = 0
    # [Options] mi = mj (a power of two) and periodic_x / periodic_y
    brick: int = 1
    periodic_x: int = 0
    periodic_y: int = 0

    def to_c(self) -> _Options:
        o = _Options()
        for name in ("mx", "my", "mbc", "meqn", "maux", "refinement_criteria", "threshold_variable",
                     "mcapa", "mwaves", "minlevel", "maxlevel", "subcycle", "regrid_interval",
                     "smooth_refine", "smooth_level", "use_fixed_dt", "nout", "init_ghostcell",
                     "reduce_cfl", "solver_kind", "problem", "step_variant", "precision", "macro_graph", "claw_version",
                     "time_sync", "weighted_partition", "ghost_fusion", "src_term", "brick", "periodic_x",
                     "periodic_y"):
            setattr(o, name, int(getattr(self, name)))
        for name in ("refine_threshold", "coarsen_threshold", "tfinal", "initial_dt", "max_cfl",
                     "desired_cfl", "grav", "gamma", "dry_tolerance"):
            setattr(o, name, float(getattr(self, name)))
        o.ax, o.bx, o.ay, o.by = (float(v) for v in self.extent)
        o.order[0], o.order[1] = int(self.order[0]), int(self.order[1])
        for k in range(8):
            o.mthlim[k] = int(self.mthlim[k]) if k < len(self.mthlim) else 0
        for k in range(4):
            o.mthbc[k] = int(self.mthbc[k])
        for k in range(32):
            o.problem_params[k] = float(self.problem_params[k]) if k < len(self.problem_params) else 0.0
        return o

    @property
    def nx(self) -> int:
        return self.mx + 2 * self.mbc

    @property
    def ny(self) -> int:
        return self.my + 2 * self.mbc


class FcbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"fcb error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load libfclaw_b200.so; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("FCB_LIBRARY", LIBPATH))
    if not path.exists():
        raise ImportError(f"{path} not found: build it with `python -m forestclaw_b200.build`")
    L = ctypes.CDLL(str(path))
    vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    sz = ctypes.c_size_t
    L.fcb_last_error.restype = ctypes.c_char_p
    L.fcb_context_create.argtypes = [ctypes.POINTER(_Options), vp, ctypes.POINTER(vp)]
    L.fcb_context_destroy.argtypes = [vp]
    for n in ("fcb_initialize", "fcb_run", "fcb_synchronize"):
        getattr(L, n).argtypes = [vp]
    L.fcb_advance_all_levels.argtypes = [vp, ctypes.c_double, ctypes.c_double, dp]
    L.fcb_advance_all_levels_async.argtypes = [vp, ctypes.c_double, ctypes.c_double]
    L.fcb_read_max_cfl.argtypes = [vp, dp]
    L.fcb_update_single_step.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, dp]
    L.fcb_update_single_step_async.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
    L.fcb_single_step_update.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_int, dp]
    L.fcb_ghost_update.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int]
    L.fcb_timeinterp.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    L.fcb_regrid.argtypes = [vp, ip]
    L.fcb_physical_set_bc.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.fcb_num_patches.argtypes = [vp, ip]
    L.fcb_patch_info.argtypes = [vp, ctypes.c_int, ip, ip, ip]
    L.fcb_patch_neighbors.argtypes = [vp, ctypes.c_int, ip]
    L.fcb_patch_size.argtypes = [vp, ctypes.POINTER(sz)]
    L.fcb_get_q.argtypes = [vp, dp, sz]
    L.fcb_set_q.argtypes = [vp, dp, sz]
    L.fcb_get_qinterp.argtypes = [vp, dp, sz]
    L.fcb_counters.argtypes = [vp, ctypes.POINTER(_Counters)]
    L.fcb_conservation_check.argtypes = [vp, dp]
    L.fcb_curr_time.argtypes = [vp, dp]
    L.fcb_autotune_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    L.fcb_step_kernel_time.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ip, dp]
    L.fcb_measure_fp_rate.argtypes = [ctypes.c_int, vp, dp]
    L.fcb_output_ascii.argtypes = [vp, ctypes.c_int, ctypes.c_char_p]
    L.fcb_conservation_sum_noalloc.argtypes = [vp, sz, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, vp, vp, vp]
    ll = ctypes.POINTER(ctypes.c_longlong)
    L.fcb_server_create.argtypes = [sz, vp, ctypes.POINTER(vp)]
    L.fcb_server_destroy.argtypes = [vp]
    L.fcb_server_submit.argtypes = [vp, ctypes.POINTER(_Options), ip]
    L.fcb_server_round.argtypes = [vp, ip, ip]
    L.fcb_server_status.argtypes = [vp, ctypes.c_int, ctypes.POINTER(RequestStatus)]
    L.fcb_server_get_q.argtypes = [vp, ctypes.c_int, dp, sz]
    L.fcb_server_release.argtypes = [vp, ctypes.c_int]
    L.fcb_server_clock.argtypes = [vp, dp, ll, ll]
    L.fcb_server_set_work_limit.argtypes = [vp, ctypes.c_longlong]
    L.fcb_comm_create_local.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.POINTER(vp)]
    L.fcb_comm_nccl_unique_id.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    L.fcb_comm_create_nccl.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, ctypes.POINTER(vp)]
    L.fcb_comm_destroy.argtypes = [vp]
    L.fcb_context_create_partitioned.argtypes = [ctypes.POINTER(_Options), vp, vp, ctypes.POINTER(vp)]
    L.fcb_partition_info.argtypes = [vp, ip, ip, ip, ip]
    L.fcb_global_maximum.argtypes = [vp, ctypes.c_double, dp]
    L.fcb_partition_plan.argtypes = [ctypes.POINTER(_Options), ctypes.c_int, ctypes.c_int, ctypes.c_int, ip, ip, ip,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int, ip, ip, ip, ip, ip, ip, ip]
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        raise FcbError(rc, lib().fcb_last_error().decode())


def measure_fp_rate(fp64: bool = True, stream: int = 0) -> float:
    """Lane add/multiply operations per second of the current GPU (FP64 or FP32)."""
    r = ctypes.c_double()
    _check(lib().fcb_measure_fp_rate(1 if fp64 else 0, ctypes.c_void_p(stream), ctypes.byref(r)))
    return r.value


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Comm:
    """One rank's communicator of a partitioned solve (fcb_comm_t)."""

    def __init__(self, handle: ctypes.c_void_p, rank: int, nranks: int):
        self._h = handle
        self.rank = rank
        self.nranks = nranks

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().fcb_comm_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def local_group(nranks: int, timeout_s: float = 120.0) -> list:
    """Communicators of an in-process group: rank r's Solver is driven by its
    own host thread (ctypes releases the GIL during library calls)."""
    arr = (ctypes.c_void_p * nranks)()
    _check(lib().fcb_comm_create_local(int(nranks), float(timeout_s), arr))
    return [Comm(ctypes.c_void_p(arr[r]), r, nranks) for r in range(nranks)]


def nccl_library() -> str:
    """libnccl.so.2 of the NCCL PyTorch ships (the one a torch process loads), else ''."""
    try:
        import nvidia.nccl as n  # noqa: PLC0415
        for root in n.__path__:
            f = Path(root) / "lib" / "libnccl.so.2"
            if f.exists():
                return str(f)
    except ImportError:
        pass
    return ""


def nccl_unique_id(library: Optional[str] = None) -> bytes:
    """The 128-byte id of a new NCCL communicator (made on one rank, sent to the others)."""
    buf = ctypes.create_string_buffer(128)
    lp = (library if library is not None else nccl_library()).encode()
    _check(lib().fcb_comm_nccl_unique_id(lp, buf))
    return buf.raw


def nccl_comm(unique_id: bytes, rank: int, nranks: int, timeout_s: float = 120.0,
              library: Optional[str] = None) -> Comm:
    """Rank `rank` of an NCCL communicator on the current CUDA device."""
    if len(unique_id) != 128:
        raise ValueError("an NCCL unique id has 128 bytes")
    h = ctypes.c_void_p()
    lp = (library if library is not None else nccl_library()).encode()
    _check(lib().fcb_comm_create_nccl(lp, unique_id, int(rank), int(nranks), float(timeout_s), ctypes.byref(h)))
    return Comm(h, rank, nranks)


def partition_plan(options: Options, leaves, rank: int, nranks: int, minlevel: int, maxlevel: int,
                   time_interp: int = 0) -> dict:
    """Host-only planning query (no GPU needed): how a partitioned solve over
    `leaves` ((level, x, y) in Morton order) splits them, and the patches each
    exchange of ghost update (minlevel, maxlevel, time_interp) sends to and
    receives from every peer rank."""
    n = len(leaves)
    lv = (ctypes.c_int * n)(*[int(l[0]) for l in leaves])
    xs = (ctypes.c_int * n)(*[int(l[1]) for l in leaves])
    ys = (ctypes.c_int * n)(*[int(l[2]) for l in leaves])
    first, count, ghosts = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    arrs = [(ctypes.c_int * nranks)() for _ in range(4)]
    copt = options.to_c()
    _check(lib().fcb_partition_plan(ctypes.byref(copt), int(nranks), int(rank), n, lv, xs, ys, int(minlevel),
                                    int(maxlevel), int(time_interp), ctypes.byref(first), ctypes.byref(count),
                                    ctypes.byref(ghosts), *arrs))
    return {"first": first.value, "count": count.value, "ghosts": ghosts.value,
            "x1_send": list(arrs[0]), "x1_recv": list(arrs[1]), "x2_send": list(arrs[2]), "x2_recv": list(arrs[3])}


class Solver:
    """One solve on one GPU (a context of the C ABI); with `comm`, one rank of
    a partitioned solve."""

    def __init__(self, options: Options, stream: Optional[int] = None, comm: Optional[Comm] = None):
        self.options = options
        self._copt = options.to_c()
        self.comm = comm
        h = ctypes.c_void_p()
        if comm is None:
            _check(lib().fcb_context_create(ctypes.byref(self._copt), ctypes.c_void_p(stream or 0),
                                            ctypes.byref(h)))
        else:
            _check(lib().fcb_context_create_partitioned(ctypes.byref(self._copt), ctypes.c_void_p(stream or 0),
                                                        comm._h, ctypes.byref(h)))
        self._h = h

    def partition_info(self) -> dict:
        """This rank, the number of ranks and the owned leaves [first, first + count)."""
        r, n, f, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().fcb_partition_info(self._h, ctypes.byref(r), ctypes.byref(n), ctypes.byref(f),
                                        ctypes.byref(c)))
        return {"rank": r.value, "nranks": n.value, "first": f.value, "count": c.value}

    def global_maximum(self, value: float) -> float:
        """fclaw2d_domain_global_maximum over the ranks of a partitioned solve."""
        out = ctypes.c_double()
        _check(lib().fcb_global_maximum(self._h, float(value), ctypes.byref(out)))
        return out.value

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().fcb_context_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- time stepping core -------------------------------------------------
    def initialize(self):
        _check(lib().fcb_initialize(self._h))

    def run(self):
        _check(lib().fcb_run(self._h))

    def advance_all_levels(self, t: float, dt: float) -> float:
        c = ctypes.c_double()
        _check(lib().fcb_advance_all_levels(self._h, t, dt, ctypes.byref(c)))
        return c.value

    def advance_all_levels_async(self, t: float, dt: float):
        """The macro step without waiting for its CFL number (see read_max_cfl)."""
        _check(lib().fcb_advance_all_levels_async(self._h, t, dt))

    def read_max_cfl(self) -> float:
        """Largest CFL number of the asynchronous macro steps since the last read."""
        c = ctypes.c_double()
        _check(lib().fcb_read_max_cfl(self._h, ctypes.byref(c)))
        return c.value

    def update_single_step(self, level: int, t: float, dt: float) -> float:
        c = ctypes.c_double()
        _check(lib().fcb_update_single_step(self._h, level, t, dt, ctypes.byref(c)))
        return c.value

    def update_single_step_async(self, level: int, t: float, dt: float):
        _check(lib().fcb_update_single_step_async(self._h, level, t, dt))

    def single_step_update(self, patchno: int, t: float, dt: float, iter: int, total_count: int) -> float:
        c = ctypes.c_double()
        _check(lib().fcb_single_step_update(self._h, patchno, t, dt, iter, total_count, ctypes.byref(c)))
        return c.value

    def ghost_update(self, minlevel: int, maxlevel: int, sync_time: float = 0.0, time_interp: int = 0):
        _check(lib().fcb_ghost_update(self._h, minlevel, maxlevel, sync_time, time_interp))

    def timeinterp(self, level: int, alpha: float):
        _check(lib().fcb_timeinterp(self._h, level, alpha))

    def regrid(self) -> bool:
        c = ctypes.c_int()
        _check(lib().fcb_regrid(self._h, ctypes.byref(c)))
        return bool(c.value)

    def physical_set_bc(self, level: int, time_interp: int = 0):
        _check(lib().fcb_physical_set_bc(self._h, level, time_interp))

    def synchronize(self):
        _check(lib().fcb_synchronize(self._h))

    # --- queries -----------------------------------------------------------
    @property
    def num_patches(self) -> int:
        n = ctypes.c_int()
        _check(lib().fcb_num_patches(self._h, ctypes.byref(n)))
        return n.value

    def patch_info(self, p: int):
        lv, x, y = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().fcb_patch_info(self._h, p, ctypes.byref(lv), ctypes.byref(x), ctypes.byref(y)))
        return lv.value, x.value, y.value

    def leaves(self):
        return [self.patch_info(p) for p in range(self.num_patches)]

    def neighbors(self, p: int):
        a = (ctypes.c_int * 22)()
        _check(lib().fcb_patch_neighbors(self._h, p, a))
        return list(a)

    def _shape(self):
        o = self.options
        if o.claw_version == 5:  # q(m,i,j): component fastest
            return (self.num_patches, o.ny, o.nx, o.meqn)
        return (self.num_patches, o.meqn, o.ny, o.nx)

    def get_q(self, out: np.ndarray | None = None) -> np.ndarray:
        """All patch arrays, (patches, meqn, ny, nx) in leaf order; `out` (for
        instance a view of pinned host memory) is filled in place if given."""
        if out is None:
            out = np.empty(self._shape(), dtype=np.float64)
        elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size < int(np.prod(self._shape())):
            raise ValueError("out must be a C-contiguous float64 array of at least the state's size")
        _check(lib().fcb_get_q(self._h, _dp(out), out.size))
        return out

    def get_qinterp(self) -> np.ndarray:
        out = np.empty(self._shape(), dtype=np.float64)
        _check(lib().fcb_get_qinterp(self._h, _dp(out), out.size))
        return out

    def set_q(self, q: np.ndarray):
        a = np.ascontiguousarray(q, dtype=np.float64)
        if a.shape != self._shape():
            raise ValueError(f"expected shape {self._shape()}, got {a.shape}")
        _check(lib().fcb_set_q(self._h, _dp(a), a.size))

    def counters(self) -> dict:
        c = _Counters()
        _check(lib().fcb_counters(self._h, ctypes.byref(c)))
        return {n: getattr(c, n) for n, _ in _Counters._fields_}

    def output_ascii(self, iframe: int, directory: str = "."):
        """Write fort.tNNNN and fort.qNNNN (the reference's ASCII frame) into `directory`."""
        _check(lib().fcb_output_ascii(self._h, int(iframe), str(directory).encode()))

    def autotune_info(self) -> dict:
        """Step form (1 CTA, 2 warp, 3 pipelined) and ghost unroll of the last launches."""
        f, u = ctypes.c_int(), ctypes.c_int()
        _check(lib().fcb_autotune_info(self._h, ctypes.byref(f), ctypes.byref(u)))
        return {"step_form": f.value, "ghost_unroll": u.value}

    def step_kernel_time(self, t: float, dt: float, launches: int = 10) -> tuple:
        """(ms per launch, fused) of the step kernel an advance launches on the
        current mesh, timed on scratch copies of the arrays."""
        f, ms = ctypes.c_int(), ctypes.c_double()
        _check(lib().fcb_step_kernel_time(self._h, t, dt, launches, ctypes.byref(f), ctypes.byref(ms)))
        return ms.value, bool(f.value)

    def conservation_check(self) -> np.ndarray:
        out = np.zeros(self.options.meqn)
        _check(lib().fcb_conservation_check(self._h, _dp(out)))
        return out

    @property
    def curr_time(self) -> float:
        t = ctypes.c_double()
        _check(lib().fcb_curr_time(self._h, ctypes.byref(t)))
        return t.value
