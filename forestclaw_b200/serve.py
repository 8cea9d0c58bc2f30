"""Ensemble serving: continuous batching of independent solves on one GPU.

Binding of the fcb_server_* entry points (include/fclaw_b200.h).  A Server
admits submitted solves while their device arrays fit its memory budget and
advances all active solves together, one fine step per round, with the patches
of every solve that shares solver, patch shape, method and precision in one
step launch.  `poisson_stream` drives it with requests that arrive at random
times (seeded), as the serving workload of the benchmark does.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np

from . import FcbError, Options, RequestStatus, _check, _dp, lib

QUEUED, ACTIVE, DONE, FAILED = 0, 1, 2, 3


class Server:
    def __init__(self, budget_bytes: int, stream: int | None = None):
        self._h = ctypes.c_void_p()
        _check(lib().fcb_server_create(int(budget_bytes), ctypes.c_void_p(stream or 0), ctypes.byref(self._h)))
        self._opts = {}

    def close(self):
        if self._h:
            lib().fcb_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, opts: Options) -> int:
        o = opts.to_c()
        rid = ctypes.c_int()
        _check(lib().fcb_server_submit(self._h, ctypes.byref(o), ctypes.byref(rid)))
        self._opts[rid.value] = opts
        return rid.value

    def set_work_limit(self, max_cells: int):
        """Admit a queued solve only while the admitted solves' cells plus its
        own stay within max_cells (0: no limit)."""
        _check(lib().fcb_server_set_work_limit(self._h, ctypes.c_longlong(int(max_cells))))

    def round(self):
        a, q = ctypes.c_int(), ctypes.c_int()
        _check(lib().fcb_server_round(self._h, ctypes.byref(a), ctypes.byref(q)))
        return a.value, q.value

    def status(self, rid: int) -> RequestStatus:
        st = RequestStatus()
        rc = lib().fcb_server_status(self._h, rid, ctypes.byref(st))
        _check(rc)
        return st

    def error(self, rid: int) -> str:
        self.status(rid)
        return lib().fcb_last_error().decode()

    def get_q(self, rid: int) -> np.ndarray:
        o = self._opts[rid]
        st = self.status(rid)
        if o.claw_version == 5:
            shape = (st.num_patches, o.ny, o.nx, o.meqn)
        else:
            shape = (st.num_patches, o.meqn, o.ny, o.nx)
        out = np.empty(shape, dtype=np.float64)
        _check(lib().fcb_server_get_q(self._h, rid, _dp(out), out.size))
        return out

    def release(self, rid: int):
        _check(lib().fcb_server_release(self._h, rid))
        self._opts.pop(rid, None)

    def clock(self):
        now, r, l = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_longlong()
        _check(lib().fcb_server_clock(self._h, ctypes.byref(now), ctypes.byref(r), ctypes.byref(l)))
        return now.value, r.value, l.value

    def run_until_idle(self, max_rounds: int = 10_000_000):
        for _ in range(max_rounds):
            a, q = self.round()
            if a == 0 and q == 0:
                return
        raise RuntimeError("server did not drain")


@dataclass
class StreamResult:
    latencies: list = field(default_factory=list)   # finish - arrival, seconds
    queue_waits: list = field(default_factory=list)  # start - arrival
    cell_updates: int = 0
    wall: float = 0.0
    rounds: int = 0
    launches: int = 0
    failed: int = 0

    def pct(self, p: float) -> float:
        return float(np.percentile(self.latencies, p)) if self.latencies else float("nan")


def poisson_stream(server: Server, requests, rate: float, seed: int = 0, keep=None) -> StreamResult:
    """Submit `requests` (Options) at Poisson arrival times of mean rate `rate`
    (per second of server clock), round until all are done, and return the
    latencies.  `keep(rid, server)` is called on each finished request before
    it is released (to collect results)."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(requests))) if rate > 0 else np.zeros(len(requests))
    res = StreamResult()
    t_base, r0, l0 = server.clock()
    pending = list(range(len(requests)))
    ids = {}
    arrival_of = {}
    live = set()
    wall0 = time.perf_counter()
    while pending or live:
        now = server.clock()[0] - t_base
        while pending and arrivals[pending[0]] <= now:
            k = pending.pop(0)
            rid = server.submit(requests[k])
            ids[rid] = k
            arrival_of[rid] = server.clock()[0]
            live.add(rid)
        if live:
            server.round()
        else:
            time.sleep(min(1e-3, max(0.0, arrivals[pending[0]] - now)))
        for rid in list(live):
            st = server.status(rid)
            if st.state in (DONE, FAILED):
                if st.state == DONE:
                    res.latencies.append(st.finish_s - arrival_of[rid])
                    res.queue_waits.append(st.start_s - arrival_of[rid])
                    res.cell_updates += st.cell_updates
                    if keep:
                        keep(ids[rid], rid, server)
                else:
                    res.failed += 1
                server.release(rid)
                live.discard(rid)
    res.wall = time.perf_counter() - wall0
    _, r1, l1 = server.clock()
    res.rounds, res.launches = r1 - r0, l1 - l0
    return res
