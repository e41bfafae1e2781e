"""ctypes mirror of ``include/frehg_gw.h`` (the C ABI of the step)."""
from __future__ import annotations

import ctypes as C
from typing import Tuple

import numpy as np

from .config import GwConfig, Rasterized, rasterize

ABI_VERSION = 1

STATUS_NAMES = {
    0: "OK", 1: "EINVAL", 2: "EUNSUPPORTED", 3: "ENOMEM", 4: "ECUDA",
    5: "ESOLVER", 6: "ENONFINITE", 7: "ESTATE",
}

FIELD = {
    "h": 0, "wc": 1, "qx": 2, "qy": 3, "qz": 4, "kx": 5, "ky": 6, "kz": 7,
    "wcn": 8, "dz3d": 9, "bot3d": 10, "ax": 11, "ay": 12, "sinx": 13, "cosx": 14,
    "siny": 15, "cosy": 16, "vloss": 17,
    "win_x": 18, "win_y": 19, "win_z": 20, "win_vent": 21,
    "rho": 22, "visc": 23, "rho_x": 24, "rho_y": 25, "rho_z": 26, "visc_x": 27, "visc_y": 28,
    "visc_z": 29, "h_prev": 30,
}
PRECISION = {"fp64": 0, "mixed": 1, "fp64_line": 2}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class GwDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double),
        ("dz_layers", _dp), ("dz_stretch", C.c_double), ("bath", _dp),
        ("follow_terrain", C.c_int), ("terrain_uniform", C.c_int),
        ("ksx", _dp), ("ksy", _dp), ("ksz", _dp), ("vg_alpha", _dp), ("vg_n", _dp),
        ("theta_s", _dp), ("theta_r", _dp), ("aev", _dp),
        ("specific_storage", C.c_double),
        ("top_code", _ip), ("bot_code", _ip), ("xm_code", _ip), ("xp_code", _ip),
        ("ym_code", _ip), ("yp_code", _ip),
        ("use_full3d", C.c_int), ("pc_consistent", C.c_int), ("face_harmonic", C.c_int),
        ("reallocation_off", C.c_int), ("surplus_redistribute", C.c_int),
        ("saturated_contact_head", C.c_int),
        ("dt_init", C.c_double), ("dt_min", C.c_double), ("dt_max", C.c_double),
        ("dq_grow", C.c_double), ("dq_shrink", C.c_double), ("courant_max", C.c_double),
        ("rtol", C.c_double), ("atol", C.c_double), ("max_iterations", C.c_int),
        ("precision", C.c_int), ("outer_rtol", C.c_double), ("max_outer", C.c_int),
    ]


class StepInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("cg_iterations", C.c_int), ("outer_iterations", C.c_int),
        ("residual_norm", C.c_double),
        ("boundary_in", C.c_double), ("ss_storage", C.c_double),
        ("realloc_adjust", C.c_double), ("realloc_dropped", C.c_double),
        ("vloss", C.c_double), ("next_dt", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


# Coupled top (include/frehg_gw.h, FREHG_GW_SURF_*).
SURF = {"eta": 0, "dept": 1, "seep_accum": 2, "avail": 3, "gain": 4, "bounce": 5, "qss": 6,
        "bottom": 7, "mode": 8}


class CoupledAudit(C.Structure):
    _fields_ = [("exchanged", C.c_double), ("bounce", C.c_double), ("vent", C.c_double),
                ("vent_thin", C.c_double), ("evap", C.c_double),
                ("pc_clamp_volume", C.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Coupling(C.Structure):
    _fields_ = [("min_depth", C.c_double), ("vent_all", C.c_int), ("book_bounce", C.c_int),
                ("field", C.c_void_p * 8)]


class Density(C.Structure):
    """frehg_gw_density: the density-coupling coefficients."""
    _fields_ = [("beta_saline", C.c_double), ("beta_saline_visc", C.c_double),
                ("thermal_expansion", C.c_double), ("reference_temperature", C.c_double),
                ("reallocation_gradient", C.c_int)]


# FREHG_GW_SCALAR_*: the density coupling's scalars.
SCALARS = {"salt": 0, "salt_surf": 1, "temp": 2, "temp_surf": 3}


class CouplerOpts(C.Structure):
    _fields_ = [("sync", C.c_int), ("dt", C.c_double), ("dt_init", C.c_double),
                ("t_start", C.c_double)]


class WindowAudit(C.Structure):
    _fields_ = [("gw", StepInfo), ("cpl", CoupledAudit), ("applied", C.c_double),
                ("discarded", C.c_double), ("surface_gain", C.c_double),
                ("accum_volume", C.c_double), ("substeps", C.c_long)]

    def as_dict(self) -> dict:
        out = {"gw": self.gw.as_dict(), "cpl": self.cpl.as_dict()}
        for name in ("applied", "discarded", "surface_gain", "accum_volume", "substeps"):
            out[name] = getattr(self, name)
        return out


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def make_desc(cfg: GwConfig, ras: Rasterized = None) -> Tuple[GwDesc, list]:
    """Fill a ``frehg_gw_desc`` from a config.  Returns the struct and the
    list of numpy buffers that must outlive the create call."""
    if ras is None:
        ras = rasterize(cfg)
    d = cfg.domain
    gw = cfg.groundwater
    s = cfg.solver
    keep = []

    def f64(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return dptr(a)

    def i32(a):
        a = np.ascontiguousarray(a, dtype=np.int32)
        keep.append(a)
        return iptr(a)

    desc = GwDesc()
    desc.abi_version = ABI_VERSION
    desc.nx, desc.ny, desc.nz = d.nx, d.ny, d.nz
    desc.dx, desc.dy = d.dx, d.dy
    desc.dz_layers = f64(ras.dz_layers)
    desc.dz_stretch = d.dz_stretch
    desc.bath = f64(ras.bath)
    desc.follow_terrain = int(bool(d.follow_terrain))
    desc.terrain_uniform = int(d.terrain_layers == "uniform")
    for name in ("ksx", "ksy", "ksz", "vg_alpha", "vg_n", "theta_s", "theta_r", "aev"):
        setattr(desc, name, f64(ras.soil[name]))
    desc.specific_storage = gw.specific_storage
    desc.top_code = i32(ras.top_code)
    desc.bot_code = i32(ras.bot_code)
    desc.xm_code = i32(ras.xm_code)
    desc.xp_code = i32(ras.xp_code)
    desc.ym_code = i32(ras.ym_code)
    desc.yp_code = i32(ras.yp_code)
    desc.use_full3d = int(bool(gw.use_full3d))
    desc.pc_consistent = int(gw.predictor_corrector == "consistent")
    desc.face_harmonic = int(gw.face_conductivity == "harmonic")
    desc.reallocation_off = int(gw.reallocation == "disabled")
    desc.surplus_redistribute = int(gw.reallocation_surplus == "redistribute")
    desc.saturated_contact_head = int(gw.saturated_contact == "head")
    ts = gw.timestep
    desc.dt_init, desc.dt_min, desc.dt_max = ts.dt_init, ts.dt_min, ts.dt_max
    desc.dq_grow, desc.dq_shrink, desc.courant_max = ts.dq_grow, ts.dq_shrink, ts.courant_max
    desc.rtol, desc.atol, desc.max_iterations = s.rtol, s.atol, s.max_iterations
    desc.precision = PRECISION[s.precision]
    desc.outer_rtol = s.outer_rtol
    desc.max_outer = s.max_outer
    return desc, keep


X_FACES = ("qx", "kx", "ax", "sinx", "cosx", "win_x", "rho_x", "visc_x")
Y_FACES = ("qy", "ky", "ay", "siny", "cosy", "win_y", "rho_y", "visc_y")
Z_FACES = ("qz", "kz", "win_z", "rho_z", "visc_z")


def field_shape(field: str, nx: int, ny: int, nz: int) -> Tuple[int, ...]:
    if field in X_FACES:
        return (ny, nx + 1, nz)
    if field in Y_FACES:
        return (ny + 1, nx, nz)
    if field in Z_FACES:
        return (ny, nx, nz + 1)
    if field == "win_vent":
        return (ny, nx)
    return (ny, nx, nz)


def interior_from_halo(field: str, full: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    """Slice a reference halo-layout field ((ny+2, nx+2, nz[+1])) to the ABI
    shape of :func:`field_shape`."""
    if field in X_FACES:
        return full[1:ny + 1, 0:nx + 1, :nz]
    if field in Y_FACES:
        return full[0:ny + 1, 1:nx + 1, :nz]
    if field in Z_FACES:
        return full[1:ny + 1, 1:nx + 1, :nz + 1]
    if field == "win_vent":
        return full[1:ny + 1, 1:nx + 1]
    return full[1:ny + 1, 1:nx + 1, :nz]
