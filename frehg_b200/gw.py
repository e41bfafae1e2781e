"""Host-side mirror of frehg2's ``gw::RichardsSolver`` over the B200 C ABI.

:class:`RichardsSolver` keeps the reference's method names and meanings
(``src/gw/RichardsSolver.hpp:166-423``): ``step(t, dtg)`` with t the
end-of-step time, ``nextDt()``, ``head()``, ``waterContent()``, the
volumetric flux accessors, ``audit()``, ``lastSolve()`` and
``ownedVolume()``.  Errors raise :class:`FatalError`, the reference's
``frehg::FatalError`` (``src/core/Types.hpp:53-62``), carrying the ABI
status.  Every call goes through ``libfrehg_gw.so`` (``include/frehg_gw.h``);
there is no CPU fallback: without the built library the constructor fails.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from .abi import (FIELD, SCALARS, STATUS_NAMES, SURF, CoupledAudit, Coupling, Density, GwDesc,
                  StepInfo, field_shape, make_desc)
from .config import IC_FORMS, GwConfig, rasterize

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfrehg_gw.so")

_dp = C.POINTER(C.c_double)
_lib = None


class FatalError(RuntimeError):
    """A non-OK status from the C ABI (reference: ``frehg::FatalError``)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load_library(path: str = LIB_PATH):
    """Load ``libfrehg_gw.so`` and declare its C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FatalError(4, f"{path} is not built; run __graft_entry__.build()")
    lib = C.CDLL(path)
    H = C.c_void_p
    lib.frehg_gw_last_error.restype = C.c_char_p
    lib.frehg_gw_create.argtypes = [C.POINTER(GwDesc), C.POINTER(H)]
    lib.frehg_gw_destroy.argtypes = [H]
    lib.frehg_gw_set_stream.argtypes = [H, C.c_void_p]
    lib.frehg_gw_set_bc_values.argtypes = [H] + [_dp] * 6
    lib.frehg_gw_init_state.argtypes = [H, C.c_int, C.c_double, _dp]
    lib.frehg_gw_set_state.argtypes = [H, _dp, _dp]
    lib.frehg_gw_restore.argtypes = [H, _dp, _dp, _dp, C.c_double]
    lib.frehg_gw_step.argtypes = [H, C.c_double, C.c_double, C.POINTER(StepInfo)]
    lib.frehg_gw_next_dt.argtypes = [H, _dp]
    lib.frehg_gw_get_field.argtypes = [H, C.c_int, _dp]
    lib.frehg_gw_field_size.argtypes = [H, C.c_int]
    lib.frehg_gw_field_size.restype = C.c_size_t
    lib.frehg_gw_owned_volume.argtypes = [H, _dp]
    lib.frehg_gw_active_cells.argtypes = [H]
    lib.frehg_gw_active_cells.restype = C.c_longlong
    lib.frehg_gw_set_profiling.argtypes = [H, C.c_int]
    lib.frehg_gw_set_profiling.restype = C.c_int
    lib.frehg_gw_phase_times.argtypes = [H, _dp]
    lib.frehg_gw_phase_times.restype = C.c_int
    lib.frehg_gw_set_fused.argtypes = [H, C.c_int]
    lib.frehg_gw_set_fused.restype = C.c_int
    lib.frehg_gw_set_warm_start.argtypes = [H, C.c_int]
    lib.frehg_gw_set_warm_start.restype = C.c_int
    lib.frehg_gw_prev_dt.argtypes = [H, _dp]
    lib.frehg_gw_prev_dt.restype = C.c_int
    lib.frehg_gw_restore_prev.argtypes = [H, _dp, C.c_double]
    lib.frehg_gw_restore_prev.restype = C.c_int
    lib.frehg_gw_kernel_launches.argtypes = [H]
    lib.frehg_gw_kernel_launches.restype = C.c_longlong
    lib.frehg_gw_attach_coupling.argtypes = [H, C.POINTER(Coupling)]
    lib.frehg_gw_get_surface.argtypes = [H, C.c_int, _dp]
    lib.frehg_gw_set_surface.argtypes = [H, C.c_int, _dp]
    lib.frehg_gw_surface_ptr.argtypes = [H, C.c_int, C.POINTER(C.c_void_p)]
    lib.frehg_gw_coupled_audit_get.argtypes = [H, C.POINTER(CoupledAudit)]
    lib.frehg_gw_elevation_offset.argtypes = [H]
    lib.frehg_gw_elevation_offset.restype = C.c_double
    lib.frehg_gw_enable_transport_window.argtypes = [H]
    lib.frehg_gw_reset_transport_window.argtypes = [H]
    lib.frehg_gw_attach_density.argtypes = [H, C.c_int, C.c_int, C.POINTER(Density)]
    lib.frehg_gw_set_scalar.argtypes = [H, C.c_int, _dp]
    lib.frehg_gw_get_scalar.argtypes = [H, C.c_int, _dp]
    lib.frehg_gw_scalar_ptr.argtypes = [H, C.c_int]
    lib.frehg_gw_scalar_ptr.restype = C.c_void_p
    for name in ("frehg_gw_create", "frehg_gw_destroy", "frehg_gw_set_stream",
                 "frehg_gw_set_bc_values", "frehg_gw_init_state", "frehg_gw_set_state",
                 "frehg_gw_step", "frehg_gw_next_dt", "frehg_gw_get_field", "frehg_gw_restore",
                 "frehg_gw_owned_volume", "frehg_gw_attach_coupling", "frehg_gw_get_surface",
                 "frehg_gw_set_surface", "frehg_gw_surface_ptr", "frehg_gw_coupled_audit_get",
                 "frehg_gw_enable_transport_window", "frehg_gw_reset_transport_window",
                 "frehg_gw_attach_density", "frehg_gw_set_scalar", "frehg_gw_get_scalar"):
        getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib


def _check(lib, rc: int):
    if rc != 0:
        raise FatalError(rc, lib.frehg_gw_last_error().decode())


class RichardsSolver:
    """The B200 groundwater step for one domain."""

    def __init__(self, cfg: GwConfig, stream: Optional[int] = None):
        self.lib = load_library()
        self.cfg = cfg
        d = cfg.domain
        self.nx, self.ny, self.nz = d.nx, d.ny, d.nz
        ras = rasterize(cfg)
        desc, keep = make_desc(cfg, ras)
        h = C.c_void_p()
        _check(self.lib, self.lib.frehg_gw_create(C.byref(desc), C.byref(h)))
        self.h = h
        if stream is not None:
            _check(self.lib, self.lib.frehg_gw_set_stream(self.h, C.c_void_p(stream)))
        self._values = [np.ascontiguousarray(v, np.float64) for v in
                        (ras.top_value, ras.bot_value, ras.xm_value, ras.xp_value,
                         ras.ym_value, ras.yp_value)]
        _check(self.lib, self.lib.frehg_gw_set_bc_values(
            self.h, *[v.ctypes.data_as(_dp) for v in self._values]))
        ic = cfg.initial
        if np.isscalar(ic.value):
            _check(self.lib, self.lib.frehg_gw_init_state(self.h, IC_FORMS[ic.form],
                                                          float(ic.value), None))
        else:
            fld = np.ascontiguousarray(ic.value, np.float64)
            _check(self.lib, self.lib.frehg_gw_init_state(self.h, IC_FORMS[ic.form], 0.0,
                                                          fld.ctypes.data_as(_dp)))
        self.t = 0.0
        self._info = None

    # -- lifetime -------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.frehg_gw_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- stepping ---------------------------------------------------------------
    def step(self, t: float, dtg: float) -> dict:
        """``RichardsSolver::step(t, dtg)``; returns the step record."""
        info = StepInfo()
        _check(self.lib, self.lib.frehg_gw_step(self.h, t, dtg, C.byref(info)))
        self._info = info.as_dict()
        return self._info

    def nextDt(self) -> float:
        out = C.c_double()
        _check(self.lib, self.lib.frehg_gw_next_dt(self.h, C.byref(out)))
        return out.value

    next_dt = nextDt

    def advance(self) -> float:
        """One adaptive step the way the reference's driver loop takes it
        (``Simulation::runGroundwaterLoop``, Simulation.cpp:1695-1700)."""
        dtg = self.nextDt()
        self.t += dtg
        self.step(self.t, dtg)
        return dtg

    def setBoundaryValues(self, top=None, bottom=None, xm=None, xp=None, ym=None, yp=None):
        """``updateBoundaryValues``: per-column / per-edge values (None keeps)."""
        arrs = [None if v is None else np.ascontiguousarray(v, np.float64)
                for v in (top, bottom, xm, xp, ym, yp)]
        _check(self.lib, self.lib.frehg_gw_set_bc_values(
            self.h, *[None if a is None else a.ctypes.data_as(_dp) for a in arrs]))

    # -- checkpoint / restart --------------------------------------------------
    def checkpoint(self) -> dict:
        """The groundwater state the reference's checkpoint stores
        (``Simulation::checkpointFields3`` and the ``dtg`` scalar,
        driver/Simulation.cpp:707-722, 1211-1216): interior h, wc, the
        cumulative clamp loss, the next dt, and the time reached."""
        ck = {"t": self.t, "dtg": self.nextDt(), "h": self.field("h"),
              "wc": self.field("wc"), "vloss": self.field("vloss")}
        # The mixed and FP64 line forms start each step from an extrapolation
        # of the last two start heads: keeping the older one makes a restart
        # take the same steps bit for bit.
        prev = C.c_double()
        _check(self.lib, self.lib.frehg_gw_prev_dt(self.h, C.byref(prev)))
        if prev.value > 0.0:
            ck["dtg_prev"] = prev.value
            ck["h_prev"] = self.field("h_prev")
        return ck

    def restore(self, ck: dict) -> None:
        """``Simulation::restoreFromCheckpoint`` for the groundwater step
        (:756-792): state, clamp-loss field and dt; the solver continues as the
        uninterrupted run would."""
        hh = np.ascontiguousarray(ck["h"], np.float64)
        ww = np.ascontiguousarray(ck["wc"], np.float64)
        vl = ck.get("vloss")
        vv = None if vl is None else np.ascontiguousarray(vl, np.float64)
        _check(self.lib, self.lib.frehg_gw_restore(
            self.h, hh.ctypes.data_as(_dp), ww.ctypes.data_as(_dp),
            None if vv is None else vv.ctypes.data_as(_dp), float(ck["dtg"])))
        if ck.get("h_prev") is not None and ck.get("dtg_prev"):
            hp = np.ascontiguousarray(ck["h_prev"], np.float64)
            _check(self.lib, self.lib.frehg_gw_restore_prev(self.h, hp.ctypes.data_as(_dp),
                                                            float(ck["dtg_prev"])))
        self.t = float(ck["t"])

    def save_checkpoint(self, path: str) -> None:
        """Writes :meth:`checkpoint` to ``path`` (numpy .npz, exact values)."""
        ck = self.checkpoint()
        extra = {"h_prev": ck["h_prev"], "dtg_prev": ck["dtg_prev"]} if "h_prev" in ck else {}
        np.savez(path, t=ck["t"], dtg=ck["dtg"], h=ck["h"], wc=ck["wc"], vloss=ck["vloss"],
                 shape=np.array([self.nx, self.ny, self.nz]), **extra)

    def load_checkpoint(self, path: str) -> None:
        with np.load(path) as z:
            if tuple(z["shape"]) != (self.nx, self.ny, self.nz):
                raise FatalError(1, f"checkpoint {path} is for a {tuple(z['shape'])} domain")
            ck = {"t": float(z["t"]), "dtg": float(z["dtg"]), "h": z["h"], "wc": z["wc"],
                  "vloss": z["vloss"]}
            if "h_prev" in z.files:
                ck["h_prev"] = z["h_prev"]
                ck["dtg_prev"] = float(z["dtg_prev"])
            self.restore(ck)

    def setState(self, head: np.ndarray, wc: np.ndarray) -> None:
        """Restart read + ``refreshDerivedState``."""
        hh = np.ascontiguousarray(head, np.float64)
        ww = np.ascontiguousarray(wc, np.float64)
        _check(self.lib, self.lib.frehg_gw_set_state(self.h, hh.ctypes.data_as(_dp),
                                                     ww.ctypes.data_as(_dp)))

    # -- observation -----------------------------------------------------------
    def field(self, name: str) -> np.ndarray:
        out = np.empty(field_shape(name, self.nx, self.ny, self.nz))
        _check(self.lib, self.lib.frehg_gw_get_field(self.h, FIELD[name],
                                                     out.ctypes.data_as(_dp)))
        return out

    def head(self) -> np.ndarray:
        return self.field("h")

    def waterContent(self) -> np.ndarray:
        return self.field("wc")

    def fluxXVolumetric(self) -> np.ndarray:
        return self.field("qx")

    def fluxYVolumetric(self) -> np.ndarray:
        return self.field("qy")

    def fluxZFaceVolumetric(self) -> np.ndarray:
        return self.field("qz")

    def audit(self) -> dict:
        """``GwStepAudit`` of the last step."""
        i = self._info or {}
        return {k: i.get(k, 0.0) for k in
                ("boundary_in", "ss_storage", "realloc_adjust", "realloc_dropped", "vloss")}

    def lastSolve(self):
        """(iterations, final preconditioned residual norm) of the last solve."""
        i = self._info or {}
        return i.get("cg_iterations", 0), i.get("residual_norm", 0.0)

    def ownedVolume(self) -> float:
        out = C.c_double()
        _check(self.lib, self.lib.frehg_gw_owned_volume(self.h, C.byref(out)))
        return out.value

    owned_volume = ownedVolume

    def activeCells(self) -> int:
        return int(self.lib.frehg_gw_active_cells(self.h))

    # -- tracing ----------------------------------------------------------------
    PHASES = ("predictor", "solve", "corrector", "post_allocation", "finalize")

    def setProfiling(self, on: bool = True) -> None:
        _check(self.lib, self.lib.frehg_gw_set_profiling(self.h, int(bool(on))))

    def setFused(self, on: bool = True) -> None:
        """Fused phase kernels (default) or every phase as separate passes."""
        _check(self.lib, self.lib.frehg_gw_set_fused(self.h, int(bool(on))))

    def setWarmStart(self, extrapolate: bool = True) -> None:
        """Mixed / FP64 line solves: start from the extrapolated head (default)
        or from h^n."""
        _check(self.lib, self.lib.frehg_gw_set_warm_start(self.h, int(bool(extrapolate))))

    def phaseTimes(self) -> dict:
        """Device ms per phase of the last step (profiling on)."""
        out = (C.c_double * 5)()
        _check(self.lib, self.lib.frehg_gw_phase_times(self.h, out))
        return dict(zip(self.PHASES, list(out)))

    def kernelLaunches(self) -> int:
        return int(self.lib.frehg_gw_kernel_launches(self.h))

    # -- coupled top (RichardsSolver::attachCoupling, RichardsSolver.hpp:132-186) --
    def attachCoupling(self, min_depth: float, vent_all: bool = False, book_bounce: bool = False,
                       device_fields: Optional[dict] = None) -> None:
        """Switches the coupled top on.  The surface fields live on the
        device, (ny+2, nx+2) each, elevations in the mesh's offset frame;
        ``device_fields`` maps names of :data:`frehg_b200.abi.SURF` to device
        addresses the caller owns, the others are allocated (zeroed)."""
        c = Coupling(float(min_depth), int(bool(vent_all)), int(bool(book_bounce)))
        for name, ptr in (device_fields or {}).items():
            c.field[SURF[name]] = int(ptr)
        _check(self.lib, self.lib.frehg_gw_attach_coupling(self.h, C.byref(c)))

    def surface(self, name: str) -> np.ndarray:
        out = np.empty((self.ny + 2, self.nx + 2))
        _check(self.lib, self.lib.frehg_gw_get_surface(self.h, SURF[name], out.ctypes.data_as(_dp)))
        return out

    def setSurface(self, name: str, value) -> None:
        v = np.ascontiguousarray(np.broadcast_to(value, (self.ny + 2, self.nx + 2)), np.float64)
        _check(self.lib, self.lib.frehg_gw_set_surface(self.h, SURF[name], v.ctypes.data_as(_dp)))

    def surfacePointer(self, name: str) -> int:
        p = C.c_void_p()
        _check(self.lib, self.lib.frehg_gw_surface_ptr(self.h, SURF[name], C.byref(p)))
        return p.value

    def couplingAudit(self) -> dict:
        """The GwStepAudit cpl* terms of the last step and pcClampVolume."""
        a = CoupledAudit()
        _check(self.lib, self.lib.frehg_gw_coupled_audit_get(self.h, C.byref(a)))
        return a.as_dict()

    def elevationOffset(self) -> float:
        return float(self.lib.frehg_gw_elevation_offset(self.h))

    # -- density coupling (RichardsSolver.hpp:191-225, Baroclinic.cpp) -----------
    def attachDensity(self, saline: bool = True, thermal: bool = False,
                      beta_saline: float = 0.000744, beta_saline_visc: float = 0.0022,
                      thermal_expansion: float = 0.0, reference_temperature: float = 20.0,
                      reallocation_gradient: bool = False) -> None:
        """attachScalar (baroclinic on) / attachTemperature /
        setDensityCoefficients: the scalars' device fields are allocated
        (zeroed); every step computes the ratios from their current values.
        Defaults are DensityCouplingConfig's."""
        d = Density(float(beta_saline), float(beta_saline_visc), float(thermal_expansion),
                    float(reference_temperature), int(bool(reallocation_gradient)))
        _check(self.lib, self.lib.frehg_gw_attach_density(self.h, int(bool(saline)),
                                                          int(bool(thermal)), C.byref(d)))

    def _scalar_shape(self, name: str):
        return ((self.ny + 2, self.nx + 2, self.nz) if SCALARS[name] in (0, 2)
                else (self.ny + 2, self.nx + 2))

    def setScalar(self, name: str, value) -> None:
        """Hand a scalar over in the halo layout (names of
        :data:`frehg_b200.abi.SCALARS`)."""
        v = np.ascontiguousarray(np.broadcast_to(value, self._scalar_shape(name)), np.float64)
        _check(self.lib, self.lib.frehg_gw_set_scalar(self.h, SCALARS[name], v.ctypes.data_as(_dp)))

    def scalar(self, name: str) -> np.ndarray:
        out = np.empty(self._scalar_shape(name))
        _check(self.lib, self.lib.frehg_gw_get_scalar(self.h, SCALARS[name], out.ctypes.data_as(_dp)))
        return out

    def scalarPointer(self, name: str) -> int:
        """Device address of a scalar field, for a producer on the device."""
        p = self.lib.frehg_gw_scalar_ptr(self.h, SCALARS[name])
        if not p:
            raise FatalError(1, f"scalar {name} not attached")
        return p

    def densityRatio(self) -> np.ndarray:
        return self.field("rho")

    def viscosityRatio(self) -> np.ndarray:
        return self.field("visc")

    def densityRatioFaceY(self) -> np.ndarray:
        return self.field("rho_y")

    def densityRatioFaceZ(self) -> np.ndarray:
        return self.field("rho_z")

    # -- transport window (RichardsSolver.hpp:229-248) ----------------------------
    def enableTransportWindow(self) -> None:
        _check(self.lib, self.lib.frehg_gw_enable_transport_window(self.h))

    def resetTransportWindow(self) -> None:
        _check(self.lib, self.lib.frehg_gw_reset_transport_window(self.h))

    def windowVolumeX(self) -> np.ndarray:
        return self.field("win_x")

    def windowVolumeY(self) -> np.ndarray:
        return self.field("win_y")

    def windowVolumeZ(self) -> np.ndarray:
        return self.field("win_z")

    def windowVentVolume(self) -> np.ndarray:
        return self.field("win_vent")
