"""Host-side mirror of frehg2's ``coupling::Coupler`` over the B200 C ABI.

:class:`Coupler` keeps the reference's method names and meanings
(``src/coupling/Coupler.hpp``): ``step(t, dt)`` advances the subsurface
through one surface step (sync: one lockstep step of dt; subcycled: every
adaptive dtg that fits, the clock lag carried over), applies the exchanged
seepage to the surface and reduces the coupled audit; ``nextDt()``,
``currentDtg()``, ``gwLag(t)``, ``restore(t, dtg, lag)``, ``audit()``,
``seepageRate()``, ``gain()`` and ``seepAccum()``.  The surface solve (the
free-surface and velocity phases, the depth refresh) is the caller's: it
runs before ``step`` on the solver's surface fields
(``RichardsSolver.surface`` / ``setSurface`` / ``surfacePointer``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .abi import CouplerOpts, WindowAudit
from .gw import RichardsSolver, _check

_dp = C.POINTER(C.c_double)


def _declare(lib):
    if getattr(lib, "_coupler_declared", False):
        return lib
    H = C.c_void_p
    lib.frehg_gw_coupler_init.argtypes = [H, C.POINTER(CouplerOpts)]
    lib.frehg_gw_coupler_step.argtypes = [H, C.c_double, C.c_double, C.POINTER(WindowAudit)]
    lib.frehg_gw_coupler_state.argtypes = [H, C.c_double, _dp, _dp, _dp]
    lib.frehg_gw_coupler_restore.argtypes = [H, C.c_double, C.c_double, C.c_double]
    for name in ("frehg_gw_coupler_init", "frehg_gw_coupler_step", "frehg_gw_coupler_state",
                 "frehg_gw_coupler_restore"):
        getattr(lib, name).restype = C.c_int
    lib._coupler_declared = True
    return lib


class Coupler:
    """The subsurface side of the coupled step for one solver (see the
    module docstring).  The solver must have its coupling attached."""

    def __init__(self, gw: RichardsSolver, sync: bool, dt: float, dt_init: float,
                 t_start: float = 0.0):
        self.gw = gw
        self.lib = _declare(gw.lib)
        o = CouplerOpts(int(bool(sync)), float(dt), float(dt_init), float(t_start))
        _check(self.lib, self.lib.frehg_gw_coupler_init(gw.h, C.byref(o)))
        self._audit = None

    def step(self, t: float, dt: float) -> dict:
        a = WindowAudit()
        _check(self.lib, self.lib.frehg_gw_coupler_step(self.gw.h, t, dt, C.byref(a)))
        self._audit = a.as_dict()
        return self._audit

    def _state(self, t: float):
        v = [C.c_double(), C.c_double(), C.c_double()]
        _check(self.lib, self.lib.frehg_gw_coupler_state(self.gw.h, t, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def nextDt(self) -> float:
        return self._state(0.0)[0]

    def currentDtg(self) -> float:
        return self._state(0.0)[1]

    def gwLag(self, t: float) -> float:
        return self._state(t)[2]

    def restore(self, t: float, dtg: float, lag: float) -> None:
        _check(self.lib, self.lib.frehg_gw_coupler_restore(self.gw.h, t, dtg, lag))

    def audit(self) -> dict:
        return self._audit

    def seepageRate(self) -> np.ndarray:
        return self.gw.surface("qss")

    def gain(self) -> np.ndarray:
        return self.gw.surface("gain")

    def seepAccum(self) -> np.ndarray:
        return self.gw.surface("seep_accum")
