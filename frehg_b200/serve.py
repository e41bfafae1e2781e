"""Serving loop for Richards solves of mixed sizes (``frehg_gw_server_*``).

``RichardsServer`` queues requests (a :class:`GwConfig` and a step count),
admits them by free device memory and slots, steps all admitted requests
together each tick (continuous batching: a request that arrives while others
are running joins at the next tick) and keeps finished results on the host.
Latency is measured from submission to completion.  :func:`run_stream` drives
a server with an arrival schedule and reports p50/p99 latency and aggregate
cell-steps/s.  The reference has no counterpart.
"""
from __future__ import annotations

import ctypes as C
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

from .abi import StepInfo, field_shape, make_desc
from .config import IC_FORMS, GwConfig, rasterize
from .gw import FatalError, load_library

_dp = C.POINTER(C.c_double)

QUEUED, RUNNING, DONE, FAILED = 0, 1, 2, 3


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("max_active", C.c_int),
                ("cells_per_block", C.c_int), ("use_graph", C.c_int), ("streams", C.c_int)]


class Request(C.Structure):
    _fields_ = [("desc", C.c_void_p), ("ic_form", C.c_int), ("ic_constant", C.c_double),
                ("ic_field", _dp), ("bc_top", _dp), ("bc_bottom", _dp), ("bc_xm", _dp),
                ("bc_xp", _dp), ("bc_ym", _dp), ("bc_yp", _dp), ("steps", C.c_int)]


class RequestStatus(C.Structure):
    _fields_ = [("state", C.c_int), ("status", C.c_int), ("steps", C.c_int),
                ("steps_done", C.c_int), ("cells", C.c_longlong), ("sim_time", C.c_double),
                ("submit_s", C.c_double), ("queue_s", C.c_double), ("latency_s", C.c_double),
                ("last", StepInfo)]


class ServerStats(C.Structure):
    _fields_ = [("active", C.c_int), ("queued", C.c_int), ("completed", C.c_longlong),
                ("ticks", C.c_longlong), ("cell_steps", C.c_longlong),
                ("device_bytes_used", C.c_size_t), ("device_bytes_budget", C.c_size_t),
                ("busy_s", C.c_double), ("now_s", C.c_double), ("admit_s", C.c_double),
                ("rebatch_s", C.c_double), ("step_s", C.c_double), ("retire_s", C.c_double)]


def _declare(lib):
    if getattr(lib, "_serve_declared", False):
        return lib
    S = C.c_void_p
    lib.frehg_gw_device_bytes.argtypes = [C.c_void_p]
    lib.frehg_gw_device_bytes.restype = C.c_size_t
    lib.frehg_gw_server_create.argtypes = [C.POINTER(ServerOpts), C.POINTER(S)]
    lib.frehg_gw_server_destroy.argtypes = [S]
    lib.frehg_gw_server_submit.argtypes = [S, C.POINTER(Request), C.POINTER(C.c_longlong)]
    lib.frehg_gw_server_tick.argtypes = [S, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.frehg_gw_server_poll.argtypes = [S, C.c_longlong, C.POINTER(RequestStatus)]
    lib.frehg_gw_server_fetch.argtypes = [S, C.c_longlong, C.c_int, _dp]
    lib.frehg_gw_server_release.argtypes = [S, C.c_longlong]
    lib.frehg_gw_server_stats.argtypes = [S, C.POINTER(ServerStats)]
    for name in ("frehg_gw_server_create", "frehg_gw_server_destroy", "frehg_gw_server_submit",
                 "frehg_gw_server_tick", "frehg_gw_server_poll", "frehg_gw_server_fetch",
                 "frehg_gw_server_release", "frehg_gw_server_stats"):
        getattr(lib, name).restype = C.c_int
    lib._serve_declared = True
    return lib


def _check(lib, rc: int):
    if rc != 0:
        raise FatalError(rc, lib.frehg_gw_last_error().decode())


class PreparedRequest:
    """A request's C structures, built once on the host (rasterised domain,
    boundary values, initial state); submitting it only copies them."""

    def __init__(self, cfg: GwConfig, steps: int):
        ras = rasterize(cfg)
        self.desc, self._keep = make_desc(cfg, ras)
        self.nx, self.ny, self.nz = cfg.domain.nx, cfg.domain.ny, cfg.domain.nz
        self._bc = [np.ascontiguousarray(v, np.float64) for v in
                    (ras.top_value, ras.bot_value, ras.xm_value, ras.xp_value, ras.ym_value,
                     ras.yp_value)]
        ic = cfg.initial
        self._field = None
        const = 0.0
        if np.isscalar(ic.value):
            const = float(ic.value)
        else:
            self._field = np.ascontiguousarray(ic.value, np.float64)
        self.req = Request(C.cast(C.pointer(self.desc), C.c_void_p), IC_FORMS[ic.form], const,
                           None if self._field is None else self._field.ctypes.data_as(_dp),
                           *[b.ctypes.data_as(_dp) for b in self._bc], int(steps))
        self.steps = steps

    def device_bytes(self) -> int:
        lib = _declare(load_library())
        return int(lib.frehg_gw_device_bytes(C.cast(C.pointer(self.desc), C.c_void_p)))


class RichardsServer:
    """See the module docstring."""

    def __init__(self, hbm_budget_bytes: int = 0, max_active: int = 0, cells_per_block: int = 0,
                 use_graph: bool = False, streams: int = 0):
        self.lib = _declare(load_library())
        opts = ServerOpts(int(hbm_budget_bytes), int(max_active), int(cells_per_block),
                          int(bool(use_graph)), int(streams))
        s = C.c_void_p()
        _check(self.lib, self.lib.frehg_gw_server_create(C.byref(opts), C.byref(s)))
        self.s = s
        self._shape: Dict[int, tuple] = {}

    def close(self) -> None:
        if getattr(self, "s", None) is not None and self.s.value:
            self.lib.frehg_gw_server_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, req, steps: Optional[int] = None) -> int:
        """Queues a request (a PreparedRequest, or a GwConfig with ``steps``)."""
        if not isinstance(req, PreparedRequest):
            req = PreparedRequest(req, steps)
        rid = C.c_longlong()
        _check(self.lib, self.lib.frehg_gw_server_submit(self.s, C.byref(req.req),
                                                         C.byref(rid)))
        self._shape[rid.value] = (req.nx, req.ny, req.nz)
        return rid.value

    def tick(self) -> tuple:
        """One admission + step + retirement round; returns (running, queued)."""
        a, q = C.c_int(), C.c_int()
        _check(self.lib, self.lib.frehg_gw_server_tick(self.s, C.byref(a), C.byref(q)))
        return a.value, q.value

    def poll(self, rid: int) -> dict:
        st = RequestStatus()
        _check(self.lib, self.lib.frehg_gw_server_poll(self.s, rid, C.byref(st)))
        out = {name: getattr(st, name) for name, _ in st._fields_ if name != "last"}
        out["last"] = st.last.as_dict()
        return out

    def result(self, rid: int) -> dict:
        """Head and water content of a finished request, (ny, nx, nz)."""
        nx, ny, nz = self._shape[rid]
        out = {}
        for name, fid in (("h", 0), ("wc", 1)):
            a = np.empty(field_shape(name, nx, ny, nz))
            _check(self.lib, self.lib.frehg_gw_server_fetch(self.s, rid, fid,
                                                            a.ctypes.data_as(_dp)))
            out[name] = a
        return out

    def release(self, rid: int) -> None:
        _check(self.lib, self.lib.frehg_gw_server_release(self.s, rid))
        self._shape.pop(rid, None)

    def stats(self) -> dict:
        st = ServerStats()
        _check(self.lib, self.lib.frehg_gw_server_stats(self.s, C.byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def run_until_idle(self, max_ticks: int = 1_000_000) -> None:
        for _ in range(max_ticks):
            a, q = self.tick()
            if a == 0 and q == 0:
                return
        raise RuntimeError("server did not drain")


def run_stream(server: RichardsServer, requests: Sequence[PreparedRequest],
               arrivals_s: Sequence[float]) -> dict:
    """Submits request i at wall time arrivals_s[i] (seconds from the start)
    while ticking the server; returns per-request latencies and totals."""
    order = np.argsort(np.asarray(arrivals_s))
    ids: List[int] = []
    t0 = time.perf_counter()
    st0 = server.stats()
    nxt = 0
    while True:
        now = time.perf_counter() - t0
        while nxt < len(order) and arrivals_s[order[nxt]] <= now:
            ids.append(server.submit(requests[order[nxt]]))
            nxt += 1
        a, q = server.tick()
        if nxt == len(order) and a == 0 and q == 0:
            break
        if a == 0 and q == 0 and nxt < len(order):
            time.sleep(max(0.0, min(arrivals_s[order[nxt]] - (time.perf_counter() - t0), 0.01)))
    wall = time.perf_counter() - t0
    st = server.stats()
    lat = []
    queue = []
    failed = 0
    for rid in ids:
        p = server.poll(rid)
        if p["state"] != DONE:
            failed += 1
        lat.append(p["latency_s"])
        queue.append(p["queue_s"])
        server.release(rid)
    lat = np.asarray(lat)
    cell_steps = st["cell_steps"] - st0["cell_steps"]
    return {"requests": len(ids), "failed": failed, "wall_s": wall,
            "cell_steps": int(cell_steps), "cell_steps_per_s": cell_steps / wall,
            "latency_p50_s": float(np.percentile(lat, 50)),
            "latency_p99_s": float(np.percentile(lat, 99)),
            "latency_max_s": float(lat.max()),
            "queue_p50_s": float(np.percentile(np.asarray(queue), 50)),
            "ticks": st["ticks"] - st0["ticks"],
            "tick_s": {k: st[k] - st0[k] for k in ("admit_s", "rebatch_s", "step_s", "retire_s")}}
