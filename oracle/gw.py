"""ctypes driver for the C restatement ``oracle/liboracle_gw.so``.

TEST INFRASTRUCTURE: the oracle is the parity checker of the B200 step.
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use it.  :class:`OracleSolver` takes the same
:class:`frehg_b200.config.GwConfig` as the product and exposes the same
method names (step, next_dt, field, owned_volume).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from frehg_b200.abi import (FIELD, SCALARS, SURF, CoupledAudit, CouplerOpts, Density, GwDesc,
                            StepInfo, WindowAudit, field_shape, make_desc)
from frehg_b200.config import IC_FORMS, GwConfig, rasterize

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_gw.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_long)
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def load():
    global _lib
    if _lib is not None:
        return _lib
    lib = C.CDLL(LIB)
    lib.oracle_gw_last_error.restype = C.c_char_p
    lib.oracle_gw_create.restype = C.c_void_p
    lib.oracle_gw_create.argtypes = [C.POINTER(GwDesc)]
    lib.oracle_gw_destroy.argtypes = [C.c_void_p]
    lib.oracle_gw_set_bc_values.argtypes = [C.c_void_p] + [_dp] * 6
    lib.oracle_gw_init_state.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp]
    lib.oracle_gw_set_state.argtypes = [C.c_void_p, _dp, _dp]
    lib.oracle_gw_step.argtypes = [C.c_void_p, C.c_double, C.c_double, C.POINTER(StepInfo)]
    lib.oracle_gw_next_dt.argtypes = [C.c_void_p]
    lib.oracle_gw_next_dt.restype = C.c_double
    lib.oracle_gw_get_field.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.oracle_gw_owned_volume.argtypes = [C.c_void_p]
    lib.oracle_gw_owned_volume.restype = C.c_double
    lib.oracle_gw_active_cells.argtypes = [C.c_void_p]
    lib.oracle_gw_active_cells.restype = C.c_longlong
    lib.oracle_gw_elevation_offset.argtypes = [C.c_void_p]
    lib.oracle_gw_elevation_offset.restype = C.c_double
    lib.oracle_gw_gid.argtypes = [C.c_void_p, _ip, _ip]
    for name in ("theta", "head", "capacity"):
        f = getattr(lib, "oracle_vg_" + name)
        f.restype = C.c_double
        f.argtypes = [C.c_double] * 6
    for name in ("conductivity", "dkdtheta"):
        f = getattr(lib, "oracle_vg_" + name)
        f.restype = C.c_double
        f.argtypes = [C.c_double] * 7
    lib.oracle_gw_last_system.restype = C.c_long
    lib.oracle_gw_last_system.argtypes = [C.c_void_p, _dp, _lp, _dp]
    lib.oracle_cg7.restype = C.c_int
    lib.oracle_cg7.argtypes = [C.c_long, _dp, _lp, _dp, _dp, C.c_double, C.c_double, C.c_int, _dp]
    lib.oracle_gw_attach_coupling.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int]
    lib.oracle_gw_surface.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
    lib.oracle_gw_coupled_audit.argtypes = [C.c_void_p, C.POINTER(CoupledAudit)]
    lib.oracle_gw_coupler_init.argtypes = [C.c_void_p, C.POINTER(CouplerOpts)]
    lib.oracle_gw_coupler_step.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp,
                                           C.POINTER(WindowAudit)]
    lib.oracle_gw_coupler_state.argtypes = [C.c_void_p, C.c_double, _dp, _dp, _dp]
    lib.oracle_gw_bath.argtypes = [C.c_void_p, _dp]
    lib.oracle_gw_enable_transport_window.argtypes = [C.c_void_p]
    lib.oracle_gw_reset_transport_window.argtypes = [C.c_void_p]
    lib.oracle_gw_window.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.oracle_gw_coupler_restore.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
    lib.oracle_gw_attach_density.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(Density)]
    lib.oracle_gw_scalar.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
    _lib = lib
    return lib


class OracleSolver:
    """The restated reference step, serial FP64 on the CPU."""

    def __init__(self, cfg: GwConfig):
        self.lib = load()
        self.cfg = cfg
        d = cfg.domain
        self.nx, self.ny, self.nz = d.nx, d.ny, d.nz
        ras = rasterize(cfg)
        desc, keep = make_desc(cfg, ras)
        h = self.lib.oracle_gw_create(C.byref(desc))
        if not h:
            raise RuntimeError("oracle create: " + self.lib.oracle_gw_last_error().decode())
        self.h = C.c_void_p(h)
        vals = [np.ascontiguousarray(v, np.float64) for v in
                (ras.top_value, ras.bot_value, ras.xm_value, ras.xp_value, ras.ym_value,
                 ras.yp_value)]
        self.lib.oracle_gw_set_bc_values(self.h, *[v.ctypes.data_as(_dp) for v in vals])
        ic = cfg.initial
        if np.isscalar(ic.value):
            rc = self.lib.oracle_gw_init_state(self.h, IC_FORMS[ic.form], float(ic.value), None)
        else:
            fld = np.ascontiguousarray(ic.value, np.float64)
            rc = self.lib.oracle_gw_init_state(self.h, IC_FORMS[ic.form], 0.0,
                                               fld.ctypes.data_as(_dp))
        if rc != 0:
            raise RuntimeError("oracle init: " + self.lib.oracle_gw_last_error().decode())
        self.t = 0.0
        self.info = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.oracle_gw_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def next_dt(self) -> float:
        return self.lib.oracle_gw_next_dt(self.h)

    def step(self, t: float, dtg: float) -> dict:
        info = StepInfo()
        rc = self.lib.oracle_gw_step(self.h, t, dtg, C.byref(info))
        if rc != 0:
            raise RuntimeError("oracle step: " + self.lib.oracle_gw_last_error().decode())
        self.info = info.as_dict()
        return self.info

    def advance(self) -> float:
        dtg = self.next_dt()
        self.t += dtg
        self.step(self.t, dtg)
        return dtg

    def field(self, name: str) -> np.ndarray:
        out = np.empty(field_shape(name, self.nx, self.ny, self.nz))
        if self.lib.oracle_gw_get_field(self.h, FIELD[name], out.ctypes.data_as(_dp)) != 0:
            raise KeyError(name)
        return out

    def set_state(self, head: np.ndarray, wc: np.ndarray) -> None:
        hh = np.ascontiguousarray(head, np.float64)
        ww = np.ascontiguousarray(wc, np.float64)
        self.lib.oracle_gw_set_state(self.h, hh.ctypes.data_as(_dp), ww.ctypes.data_as(_dp))

    def last_system(self):
        """(vals7, cols7, rhs) of the last predictor system."""
        n = self.active_cells()
        v = np.empty((n, 7))
        c = np.empty((n, 7), dtype=np.int64)
        b = np.empty(n)
        self.lib.oracle_gw_last_system(self.h, v.ctypes.data_as(_dp), c.ctypes.data_as(_lp),
                                       b.ctypes.data_as(_dp))
        return v, c, b

    def owned_volume(self) -> float:
        return self.lib.oracle_gw_owned_volume(self.h)

    def active_cells(self) -> int:
        return self.lib.oracle_gw_active_cells(self.h)

    def elevation_offset(self) -> float:
        return self.lib.oracle_gw_elevation_offset(self.h)

    def set_boundary_values(self, top=None, bottom=None, xm=None, xp=None, ym=None, yp=None):
        """updateBoundaryValues: per-column / per-edge values (None keeps)."""
        arrs = [None if v is None else np.ascontiguousarray(v, np.float64)
                for v in (top, bottom, xm, xp, ym, yp)]
        self._check(self.lib.oracle_gw_set_bc_values(
            self.h, *[None if a is None else a.ctypes.data_as(_dp) for a in arrs]))

    # ------------------------------------------------------------ density coupling
    def attach_density(self, saline: bool = True, thermal: bool = False,
                       beta_saline: float = 0.000744, beta_saline_visc: float = 0.0022,
                       thermal_expansion: float = 0.0, reference_temperature: float = 20.0,
                       reallocation_gradient: bool = False) -> None:
        d = Density(beta_saline, beta_saline_visc, thermal_expansion, reference_temperature,
                    int(reallocation_gradient))
        self._check(self.lib.oracle_gw_attach_density(self.h, int(saline), int(thermal),
                                                      C.byref(d)))

    def _scalar_shape(self, which):
        return ((self.ny + 2, self.nx + 2, self.nz) if SCALARS[which] in (0, 2)
                else (self.ny + 2, self.nx + 2))

    def scalar(self, which: str) -> np.ndarray:
        out = np.empty(self._scalar_shape(which))
        self._check(self.lib.oracle_gw_scalar(self.h, SCALARS[which], out.ctypes.data_as(_dp),
                                              None))
        return out

    def set_scalar(self, which: str, value) -> None:
        v = np.ascontiguousarray(np.broadcast_to(value, self._scalar_shape(which)), np.float64)
        self._check(self.lib.oracle_gw_scalar(self.h, SCALARS[which], None,
                                              v.ctypes.data_as(_dp)))

    # ------------------------------------------------------------ coupled top
    def attach_coupling(self, min_depth: float, vent_all: bool = False,
                        book_bounce: bool = False) -> None:
        self._check(self.lib.oracle_gw_attach_coupling(self.h, min_depth, int(vent_all),
                                                       int(book_bounce)))

    def surface(self, name: str) -> np.ndarray:
        out = np.empty((self.ny + 2, self.nx + 2))
        self._check(self.lib.oracle_gw_surface(self.h, SURF[name], out.ctypes.data_as(_dp),
                                               None))
        return out

    def set_surface(self, name: str, value) -> None:
        v = np.ascontiguousarray(np.broadcast_to(value, (self.ny + 2, self.nx + 2)), np.float64)
        self._check(self.lib.oracle_gw_surface(self.h, SURF[name], None, v.ctypes.data_as(_dp)))

    def coupled_audit(self) -> dict:
        a = CoupledAudit()
        self.lib.oracle_gw_coupled_audit(self.h, C.byref(a))
        return a.as_dict()

    def coupler_init(self, sync: bool, dt: float, dt_init: float, t_start: float = 0.0) -> None:
        o = CouplerOpts(int(sync), dt, dt_init, t_start)
        self._check(self.lib.oracle_gw_coupler_init(self.h, C.byref(o)))

    def coupler_step(self, t: float, dt: float, bottom: np.ndarray) -> dict:
        b = np.ascontiguousarray(bottom, np.float64)
        a = WindowAudit()
        self._check(self.lib.oracle_gw_coupler_step(self.h, t, dt, b.ctypes.data_as(_dp),
                                                    C.byref(a)))
        return a.as_dict()

    def coupler_state(self, t: float) -> tuple:
        v = [C.c_double(), C.c_double(), C.c_double()]
        self.lib.oracle_gw_coupler_state(self.h, t, *[C.byref(x) for x in v])
        return tuple(x.value for x in v)

    def coupler_restore(self, t: float, dtg: float, lag: float) -> None:
        self.lib.oracle_gw_coupler_restore(self.h, t, dtg, lag)

    # ------------------------------------------------------------ transport window
    WINDOWS = {"x": 0, "y": 1, "z": 2, "vent": 3}

    def enable_transport_window(self) -> None:
        self._check(self.lib.oracle_gw_enable_transport_window(self.h))

    def reset_transport_window(self) -> None:
        self.lib.oracle_gw_reset_transport_window(self.h)

    def window(self, name: str) -> np.ndarray:
        """Window volumes in the halo layouts ((ny+2, nx+2, nz[+1]) or
        (ny+2, nx+2) for the vent)."""
        nzf = self.nz + 1 if name == "z" else self.nz
        shape = (self.ny + 2, self.nx + 2) if name == "vent" else (self.ny + 2, self.nx + 2, nzf)
        out = np.empty(shape)
        self._check(self.lib.oracle_gw_window(self.h, self.WINDOWS[name], out.ctypes.data_as(_dp)))
        return out

    def bath_halo(self) -> np.ndarray:
        """The mesh bed, offset frame, (ny+2, nx+2) with the mirrored halo."""
        out = np.empty((self.ny + 2, self.nx + 2))
        self.lib.oracle_gw_bath(self.h, out.ctypes.data_as(_dp))
        return out

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise RuntimeError("oracle: " + self.lib.oracle_gw_last_error().decode())

    def gid(self):
        gid = np.empty((self.ny + 2, self.nx + 2, self.nz), np.int32)
        ktop = np.empty((self.ny, self.nx), np.int32)
        self.lib.oracle_gw_gid(self.h, gid.ctypes.data_as(_ip), ktop.ctypes.data_as(_ip))
        return gid, ktop


def vg(name: str, soil, *args) -> float:
    """Evaluate one oracle closure: soil = (alpha, n, theta_s, theta_r, aev)."""
    return getattr(load(), "oracle_vg_" + name)(*soil, *args)
