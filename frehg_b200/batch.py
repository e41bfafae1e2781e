"""Many independent groundwater domains stepped together (``frehg_gw_batch_*``).

``RichardsBatch`` is a view over existing :class:`frehg_b200.gw.RichardsSolver`
objects: each batch step advances every member by its own adaptive dt, the
way ``RichardsSolver.advance`` does: each non-solve phase is one launch for
all members (or, with ``per_member_phases``, member by member on concurrent
streams), their predictor solves one cooperative launch per kernel class, and
the whole step is replayed from a CUDA graph.  Members remain ordinary solvers
between steps (boundary values, fields, state).  The reference has no
counterpart: its driver steps one domain per rank.
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, List, Optional

from .abi import StepInfo
from .gw import FatalError, RichardsSolver, load_library


class BatchOpts(C.Structure):
    _fields_ = [("cells_per_block", C.c_int), ("tiled_line_solve", C.c_int),
                ("use_graph", C.c_int), ("streams", C.c_int), ("per_member_phases", C.c_int)]


class BatchStats(C.Structure):
    _fields_ = [("members", C.c_int), ("solve_launches", C.c_int), ("solve_blocks", C.c_int),
                ("graphs", C.c_int), ("uses_graph", C.c_int), ("steps", C.c_longlong),
                ("kernel_launches", C.c_longlong), ("kernels_per_step", C.c_longlong),
                ("cells_per_block", C.c_int), ("tiled_line_solve", C.c_int),
                ("phase_ms", C.c_double * 3)]


def _declare(lib):
    if getattr(lib, "_batch_declared", False):
        return lib
    H, B = C.c_void_p, C.c_void_p
    lib.frehg_gw_batch_create.argtypes = [C.POINTER(C.c_void_p), C.c_int,
                                          C.POINTER(BatchOpts), C.POINTER(B)]
    lib.frehg_gw_batch_destroy.argtypes = [B]
    lib.frehg_gw_batch_step.argtypes = [B, C.POINTER(StepInfo)]
    lib.frehg_gw_batch_set_dt.argtypes = [B, C.c_int, C.c_double]
    lib.frehg_gw_batch_autotune.argtypes = [B, C.c_int, C.POINTER(BatchOpts),
                                            C.POINTER(C.c_double)]
    lib.frehg_gw_batch_stats.argtypes = [B, C.POINTER(BatchStats)]
    lib.frehg_gw_batch_solve_blocks.argtypes = [B, C.POINTER(C.c_int)]
    lib.frehg_gw_batch_set_members.argtypes = [B, C.POINTER(C.c_void_p), C.c_int]
    for name in ("frehg_gw_batch_create", "frehg_gw_batch_destroy", "frehg_gw_batch_step",
                 "frehg_gw_batch_set_dt", "frehg_gw_batch_autotune", "frehg_gw_batch_stats",
                 "frehg_gw_batch_solve_blocks", "frehg_gw_batch_set_members"):
        getattr(lib, name).restype = C.c_int
    del H
    lib._batch_declared = True
    return lib


def _check(lib, rc: int):
    if rc != 0:
        raise FatalError(rc, lib.frehg_gw_last_error().decode())


class RichardsBatch:
    """Steps the given solvers together; see the module docstring."""

    def __init__(self, solvers: Iterable[RichardsSolver], cells_per_block: int = 0,
                 tiled_line_solve: bool = False, use_graph: bool = True, streams: int = 0,
                 per_member_phases: bool = False):
        self.lib = _declare(load_library())
        self.members: List[RichardsSolver] = list(solvers)
        n = len(self.members)
        arr = (C.c_void_p * n)(*[s.h.value for s in self.members])
        opts = BatchOpts(int(cells_per_block), int(bool(tiled_line_solve)), int(bool(use_graph)),
                         int(streams), int(bool(per_member_phases)))
        b = C.c_void_p()
        _check(self.lib, self.lib.frehg_gw_batch_create(arr, n, C.byref(opts), C.byref(b)))
        self.b = b

    def __len__(self) -> int:
        return len(self.members)

    def close(self) -> None:
        if getattr(self, "b", None) is not None and self.b.value:
            self.lib.frehg_gw_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def step(self) -> List[dict]:
        """One adaptive step of every member; returns their step records."""
        n = len(self.members)
        dts = [s.nextDt() for s in self.members]
        infos = (StepInfo * n)()
        rc = self.lib.frehg_gw_batch_step(self.b, infos)
        out = [infos[i].as_dict() for i in range(n)]
        for s, dt, info in zip(self.members, dts, out):
            if info["status"] == 0:
                s.t += dt
                s._info = info
        _check(self.lib, rc)
        return out

    def set_members(self, solvers: Iterable[RichardsSolver]) -> None:
        """Rebinds the batch to a new member list, reusing its buffers."""
        self.members = list(solvers)
        n = len(self.members)
        arr = (C.c_void_p * n)(*[s.h.value for s in self.members])
        _check(self.lib, self.lib.frehg_gw_batch_set_members(self.b, arr, n))

    def set_dt(self, i: int, dtg: float) -> None:
        _check(self.lib, self.lib.frehg_gw_batch_set_dt(self.b, i, dtg))

    def autotune(self, trials: int = 1) -> tuple:
        """Picks the decomposition; returns (options dict, best step ms or -1)."""
        chosen = BatchOpts()
        best = C.c_double()
        _check(self.lib, self.lib.frehg_gw_batch_autotune(self.b, trials, C.byref(chosen),
                                                          C.byref(best)))
        return ({"cells_per_block": chosen.cells_per_block,
                 "tiled_line_solve": bool(chosen.tiled_line_solve)}, best.value)

    def stats(self) -> dict:
        st = BatchStats()
        _check(self.lib, self.lib.frehg_gw_batch_stats(self.b, C.byref(st)))
        out = {name: getattr(st, name) for name, _ in st._fields_}
        out["phase_ms"] = list(st.phase_ms)
        return out

    def solve_blocks(self) -> List[int]:
        n = len(self.members)
        nb = (C.c_int * n)()
        _check(self.lib, self.lib.frehg_gw_batch_solve_blocks(self.b, nb))
        return list(nb)


def open_batch(cfgs, **opts) -> Optional[RichardsBatch]:
    """Creates one solver per config and a batch over them."""
    solvers = [RichardsSolver(c) for c in cfgs]
    return RichardsBatch(solvers, **opts)
