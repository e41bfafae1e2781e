"""Driver for the reference's own groundwater step (test infrastructure).

``oracle/_ref/libfrehg_ref.so`` is the reference's unmodified ``src/gw``,
``src/core``, ``src/bc`` and ``src/io`` sources compiled against the host
shims in ``oracle/shim`` (recipe: ``oracle/Makefile``, target ``ref``).
:class:`RefSolver` builds a ``frehg::gw::RichardsSolver`` the way the
reference's unit tests do (``tests/unit/test_gw.cpp:33-61``) and exposes its
fields in the ABI shapes of ``include/frehg_gw.h``.  Used only by tests and
by the CPU-baseline leg of ``bench.py``.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
from typing import Optional

import numpy as np

from frehg_b200.abi import SCALARS, interior_from_halo
from frehg_b200.config import GwConfig

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_SERIAL = os.path.join(HERE, "_ref", "libfrehg_ref.so")
LIB_OMP = os.path.join(HERE, "_ref", "libfrehg_ref_omp.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class RefCase(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dz_stretch", C.c_double),
        ("follow_terrain", C.c_int), ("terrain_uniform", C.c_int),
        ("bath", _dp), ("n_soil_types", C.c_int), ("soil_types", _dp), ("soil_map", _ip),
        ("ic_form", C.c_int), ("ic_const", C.c_double), ("ic_field", _dp),
        ("ss", C.c_double),
        ("use_full3d", C.c_int), ("pc_consistent", C.c_int), ("harmonic", C.c_int),
        ("realloc_off", C.c_int), ("surplus_redistribute", C.c_int), ("sc_head", C.c_int),
        ("dt_init", C.c_double), ("dt_min", C.c_double), ("dt_max", C.c_double),
        ("dq_grow", C.c_double), ("dq_shrink", C.c_double), ("courant_max", C.c_double),
        ("rtol", C.c_double), ("atol", C.c_double), ("maxit", C.c_int),
        ("n_bc", C.c_int), ("bc_target", _ip), ("bc_kind", _ip), ("bc_form", _ip),
        ("bc_value", _dp), ("bc_eta", _dp), ("bc_npts", _ip), ("bc_pts", _dp),
        ("workdir", C.c_char_p), ("pc", C.c_char_p),
    ]


_libs = {}


def available(omp: bool = False) -> bool:
    return os.path.exists(LIB_OMP if omp else LIB_SERIAL)


def load(omp: bool = False):
    path = LIB_OMP if omp else LIB_SERIAL
    if path in _libs:
        return _libs[path]
    lib = C.CDLL(path)
    lib.ref_create.restype = C.c_void_p
    lib.ref_create.argtypes = [C.POINTER(RefCase)]
    lib.ref_last_error.restype = C.c_char_p
    lib.ref_destroy.argtypes = [C.c_void_p]
    lib.ref_step.argtypes = [C.c_void_p, C.c_double, C.c_double]
    lib.ref_step.restype = C.c_int
    lib.ref_next_dt.argtypes = [C.c_void_p]
    lib.ref_next_dt.restype = C.c_double
    lib.ref_owned_volume.argtypes = [C.c_void_p]
    lib.ref_owned_volume.restype = C.c_double
    lib.ref_audit.argtypes = [C.c_void_p, _dp]
    lib.ref_last_solve.argtypes = [C.c_void_p, _ip, _dp]
    lib.ref_elevation_offset.argtypes = [C.c_void_p]
    lib.ref_elevation_offset.restype = C.c_double
    lib.ref_get.argtypes = [C.c_void_p, C.c_char_p, _dp]
    lib.ref_get.restype = C.c_int
    lib.ref_set_state.argtypes = [C.c_void_p, _dp, _dp]
    lib.ref_gid.argtypes = [C.c_void_p, _ip, _ip]
    lib.ref_bc_masks.argtypes = [C.c_void_p, C.c_double, _ip, _dp]
    lib.ref_reallocate_only.argtypes = [C.c_void_p]
    lib.ref_attach_coupling.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int]
    lib.ref_surface.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
    lib.ref_coupled_audit.argtypes = [C.c_void_p, _dp]
    lib.ref_coupler_create.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_int]
    lib.ref_coupler_step.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp]
    lib.ref_coupler_state.argtypes = [C.c_void_p, C.c_double, _dp]
    lib.ref_enable_transport_window.argtypes = [C.c_void_p]
    lib.ref_reset_transport_window.argtypes = [C.c_void_p]
    lib.ref_window.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.ref_attach_density.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double,
                                       C.c_double, C.c_double, C.c_int]
    lib.ref_scalar.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
    _libs[path] = lib
    return lib


_TARGET = {"groundwater_top": 1, "groundwater_bottom": 2, "groundwater_side": 3}
_KIND = {"head": 4, "flux": 5}
_FORM = {"constant": 0, "gravity": 2, "hydrostatic": 3}
_IC = {"moisture": 0, "head": 1, "water_table": 2}

AUDIT_KEYS = ("boundary_in", "ss_storage", "realloc_adjust", "realloc_dropped", "vloss",
              "cpl_vent", "pc_clamp_volume")
CPL_KEYS = ("exchanged", "bounce", "vent", "vent_thin", "evap", "pc_clamp_volume")
WINDOW_GW_KEYS = ("boundary_in", "ss_storage", "realloc_adjust", "realloc_dropped", "vloss")
# ref_surface slots: the FREHG_GW_SURF_* numbering, plus the stand-in's rain.
SURF = {"eta": 0, "dept": 1, "seep_accum": 2, "avail": 3, "gain": 4, "bounce": 5, "qss": 6,
        "bottom": 7, "rain": 9}


class RefSolver:
    """The reference ``RichardsSolver`` on the CPU (serial, or OpenMP shim)."""

    def __init__(self, cfg: GwConfig, pc: str = "jacobi", omp: bool = False,
                 workdir: Optional[str] = None):
        self.lib = load(omp)
        self.cfg = cfg
        d = cfg.domain
        self.nx, self.ny, self.nz = d.nx, d.ny, d.nz
        self._tmp = tempfile.TemporaryDirectory(prefix="frehg_ref_") if workdir is None else None
        wd = workdir or self._tmp.name
        keep = []

        def f64(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return a.ctypes.data_as(_dp)

        def i32(a):
            a = np.ascontiguousarray(a, dtype=np.int32)
            keep.append(a)
            return a.ctypes.data_as(_ip)

        c = RefCase()
        c.nx, c.ny, c.nz = d.nx, d.ny, d.nz
        c.dx, c.dy, c.dz, c.dz_stretch = d.dx, d.dy, d.dz, d.dz_stretch
        c.follow_terrain = int(bool(d.follow_terrain))
        c.terrain_uniform = int(d.terrain_layers == "uniform")
        if np.isscalar(d.bottom_elevation):
            c.bath = f64(np.full(d.ny * d.nx, float(d.bottom_elevation)))
        else:
            c.bath = f64(np.asarray(d.bottom_elevation).reshape(-1))
        cols = ("ksx", "ksy", "ksz", "theta_s", "theta_r", "vg_alpha", "vg_n", "aev")
        if cfg.cell_soil is not None and cfg.soil_map is None:
            # Per-cell soil reaches the reference the only way it takes it:
            # one soil type per cell and the id map 0..ncell-1 in the
            # reference's (j*nx + i)*nz + k order.  Built from the arrays
            # directly (a 512x512x128 slab has 33.5M types).
            ncell = d.nx * d.ny * d.nz
            base = cfg.soil_types[0]
            st = np.empty((ncell, 8), dtype=np.float64)
            for n, name in enumerate(cols):
                v = cfg.cell_soil.get(name, getattr(base, name))
                st[:, n] = np.broadcast_to(np.asarray(v, np.float64),
                                           (d.ny, d.nx, d.nz)).reshape(-1)
            c.n_soil_types = ncell
            c.soil_types = f64(st.reshape(-1))
            c.soil_map = i32(np.arange(ncell, dtype=np.int32))
        else:
            st = np.array([[getattr(s, name) for name in cols] for s in cfg.soil_types],
                          dtype=np.float64)
            c.n_soil_types = len(cfg.soil_types)
            c.soil_types = f64(st.reshape(-1))
            c.soil_map = (i32(np.asarray(cfg.soil_map).reshape(-1))
                          if cfg.soil_map is not None else None)
        ic = cfg.initial
        c.ic_form = _IC[ic.form]
        if np.isscalar(ic.value):
            c.ic_const = float(ic.value)
            c.ic_field = None
        else:
            c.ic_field = f64(np.asarray(ic.value).reshape(-1))
        gw = cfg.groundwater
        c.ss = gw.specific_storage
        c.use_full3d = int(bool(gw.use_full3d))
        c.pc_consistent = int(gw.predictor_corrector == "consistent")
        c.harmonic = int(gw.face_conductivity == "harmonic")
        c.realloc_off = int(gw.reallocation == "disabled")
        c.surplus_redistribute = int(gw.reallocation_surplus == "redistribute")
        c.sc_head = int(gw.saturated_contact == "head")
        ts = gw.timestep
        c.dt_init, c.dt_min, c.dt_max = ts.dt_init, ts.dt_min, ts.dt_max
        c.dq_grow, c.dq_shrink, c.courant_max = ts.dq_grow, ts.dq_shrink, ts.courant_max
        c.rtol, c.atol, c.maxit = cfg.solver.rtol, cfg.solver.atol, cfg.solver.max_iterations
        bcs = cfg.boundary_conditions
        c.n_bc = len(bcs)
        if bcs:
            c.bc_target = i32([_TARGET[b.target] for b in bcs])
            c.bc_kind = i32([_KIND[b.kind] for b in bcs])
            c.bc_form = i32([_FORM[b.form] for b in bcs])
            c.bc_value = f64([b.value for b in bcs])
            c.bc_eta = f64([b.hydrostatic_eta for b in bcs])
            c.bc_npts = i32([len(b.polygon) for b in bcs])
            c.bc_pts = f64(np.array([p for b in bcs for p in b.polygon], dtype=np.float64).reshape(-1))
        c.workdir = wd.encode()
        c.pc = pc.encode()
        h = self.lib.ref_create(C.byref(c))
        if not h:
            raise RuntimeError("reference RichardsSolver: " + self.lib.ref_last_error().decode())
        self.h = C.c_void_p(h)
        self.t = 0.0

    def close(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- stepping (MiniGw::step, test_gw.cpp:53-58) -------------------------
    def next_dt(self) -> float:
        return self.lib.ref_next_dt(self.h)

    def step(self, t: float, dtg: float) -> None:
        if self.lib.ref_step(self.h, t, dtg) != 0:
            raise RuntimeError("reference step: " + self.lib.ref_last_error().decode())

    def advance(self) -> float:
        dtg = self.next_dt()
        self.t += dtg
        self.step(self.t, dtg)
        return dtg

    # -- observation -----------------------------------------------------------
    def _halo_shape(self, name):
        nz = self.nz + 1 if name in ("qz", "kz", "rho_z") else self.nz
        return (self.ny + 2, self.nx + 2, nz)

    def halo_field(self, name: str) -> np.ndarray:
        if name == "bath":
            out = np.empty((self.ny + 2, self.nx + 2))
        else:
            out = np.empty(self._halo_shape(name))
        if self.lib.ref_get(self.h, name.encode(), out.ctypes.data_as(_dp)) != 0:
            raise KeyError(name)
        return out

    def field(self, name: str) -> np.ndarray:
        return np.ascontiguousarray(
            interior_from_halo(name, self.halo_field(name), self.nx, self.ny, self.nz))

    def audit(self) -> dict:
        out = np.zeros(7)
        self.lib.ref_audit(self.h, out.ctypes.data_as(_dp))
        return dict(zip(AUDIT_KEYS, out.tolist()))

    def last_solve(self):
        it = C.c_int()
        res = C.c_double()
        self.lib.ref_last_solve(self.h, C.byref(it), C.byref(res))
        return it.value, res.value

    def owned_volume(self) -> float:
        return self.lib.ref_owned_volume(self.h)

    def elevation_offset(self) -> float:
        return self.lib.ref_elevation_offset(self.h)

    def gid(self):
        gid = np.empty((self.ny + 2, self.nx + 2, self.nz), np.int32)
        ktop = np.empty((self.ny, self.nx), np.int32)
        self.lib.ref_gid(self.h, gid.ctypes.data_as(_ip), ktop.ctypes.data_as(_ip))
        return gid, ktop

    def bc_masks(self, t: float = 0.0):
        n2 = (self.ny + 2) * (self.nx + 2)
        codes = np.zeros(6 * n2, np.int32)
        vals = np.zeros(6 * n2)
        self.lib.ref_bc_masks(self.h, t, codes.ctypes.data_as(_ip), vals.ctypes.data_as(_dp))
        return (codes.reshape(6, self.ny + 2, self.nx + 2), vals.reshape(6, self.ny + 2, self.nx + 2))

    def set_state_interior(self, head: np.ndarray, wc: np.ndarray) -> None:
        hf = self.halo_field("h")
        wf = self.halo_field("wc")
        hf[1:-1, 1:-1, :] = head
        wf[1:-1, 1:-1, :] = wc
        self.lib.ref_set_state(self.h, hf.ctypes.data_as(_dp), wf.ctypes.data_as(_dp))

    # -- coupled top -------------------------------------------------------------
    def attach_coupling(self, min_depth: float, vent_all: bool = False,
                        book_bounce: bool = False) -> None:
        """Harness-owned GwCoupling views, zeroed (Coupler.cpp:40-60)."""
        self.lib.ref_attach_coupling(self.h, min_depth, int(vent_all), int(book_bounce))

    def surface(self, name: str) -> np.ndarray:
        out = np.empty((self.ny + 2, self.nx + 2))
        if self.lib.ref_surface(self.h, SURF[name], out.ctypes.data_as(_dp), None) != 0:
            raise KeyError(name)
        return out

    def set_surface(self, name: str, value) -> None:
        v = np.ascontiguousarray(np.broadcast_to(value, (self.ny + 2, self.nx + 2)), np.float64)
        if self.lib.ref_surface(self.h, SURF[name], None, v.ctypes.data_as(_dp)) != 0:
            raise KeyError(name)

    def coupled_audit(self) -> dict:
        out = np.zeros(6)
        self.lib.ref_coupled_audit(self.h, out.ctypes.data_as(_dp))
        return dict(zip(CPL_KEYS, out.tolist()))

    def coupler_create(self, sync: bool, dt: float, dt_init: float, t_start: float = 0.0,
                       min_depth: float = 0.0, paired: bool = False) -> None:
        """The reference's coupling::Coupler over the stand-in surface
        (oracle/shim/include/swe/SurfaceSolver.hpp)."""
        if self.lib.ref_coupler_create(self.h, int(sync), dt, dt_init, t_start, min_depth,
                                       int(paired)) != 0:
            raise RuntimeError("reference Coupler: " + self.lib.ref_last_error().decode())

    def coupler_step(self, t: float, dt: float) -> dict:
        out = np.zeros(15)
        if self.lib.ref_coupler_step(self.h, t, dt, out.ctypes.data_as(_dp)) != 0:
            raise RuntimeError("reference coupled step: " + self.lib.ref_last_error().decode())
        v = out.tolist()
        return {"gw": dict(zip(WINDOW_GW_KEYS, v[:5])), "cpl": dict(zip(CPL_KEYS[:5], v[5:10])),
                "applied": v[10], "discarded": v[11], "surface_gain": v[12],
                "accum_volume": v[13], "substeps": int(v[14])}

    def coupler_state(self, t: float) -> tuple:
        out = np.zeros(3)
        self.lib.ref_coupler_state(self.h, t, out.ctypes.data_as(_dp))
        return tuple(out.tolist())

    # -- transport window --------------------------------------------------------
    WINDOWS = {"x": 0, "y": 1, "z": 2, "vent": 3}

    def enable_transport_window(self) -> None:
        self.lib.ref_enable_transport_window(self.h)

    def reset_transport_window(self) -> None:
        self.lib.ref_reset_transport_window(self.h)

    def window(self, name: str) -> np.ndarray:
        """Window volumes in the halo layouts ((ny+2, nx+2, nz[+1]) or
        (ny+2, nx+2) for the vent)."""
        shape = {"x": self._halo_shape("qx"), "y": self._halo_shape("qy"),
                 "z": self._halo_shape("qz"), "vent": (self.ny + 2, self.nx + 2)}[name]
        out = np.empty(shape)
        if self.lib.ref_window(self.h, self.WINDOWS[name], out.ctypes.data_as(_dp)) != 0:
            raise KeyError(name)
        return out

    # -- density coupling ---------------------------------------------------------
    def attach_density(self, saline: bool = True, thermal: bool = False,
                       beta_saline: float = 0.000744, beta_saline_visc: float = 0.0022,
                       thermal_expansion: float = 0.0, reference_temperature: float = 20.0,
                       reallocation_gradient: bool = False) -> None:
        """attachScalar (baroclinic on) / attachTemperature /
        setDensityCoefficients with harness-owned scalar views, zeroed."""
        self.lib.ref_attach_density(self.h, int(saline), int(thermal), beta_saline,
                                    beta_saline_visc, thermal_expansion, reference_temperature,
                                    int(reallocation_gradient))

    def _scalar_shape(self, which):
        return ((self.ny + 2, self.nx + 2, self.nz) if SCALARS[which] in (0, 2)
                else (self.ny + 2, self.nx + 2))

    def scalar(self, which: str) -> np.ndarray:
        out = np.empty(self._scalar_shape(which))
        if self.lib.ref_scalar(self.h, SCALARS[which], out.ctypes.data_as(_dp), None) != 0:
            raise KeyError(which)
        return out

    def set_scalar(self, which: str, value) -> None:
        v = np.ascontiguousarray(np.broadcast_to(value, self._scalar_shape(which)), np.float64)
        if self.lib.ref_scalar(self.h, SCALARS[which], None, v.ctypes.data_as(_dp)) != 0:
            raise KeyError(which)
