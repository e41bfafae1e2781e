"""Miniature groundwater cases shared by the test modules.

Each builder reproduces one configuration of the reference's groundwater
unit tests (``tests/unit/test_gw.cpp``), which assemble a ``FrehgConfig`` in
code (``gwBaseConfig`` :86-109, ``testSoil`` :71-84, ``topBc`` :131-141).
"""
from __future__ import annotations

import math

import numpy as np

from frehg_b200.config import (BoundaryCondition, Domain, Groundwater, GwConfig,
                               InitialCondition, Solver, SoilType, Timestep, whole_footprint)


def test_soil(ks: float = 1.0e-5, name: str = "test") -> SoilType:
    """``testSoil`` (test_gw.cpp:71-84): sand-shaped retention, slow Ks."""
    return SoilType(name, ks, ks, ks, 0.46, 0.04, 5.9, 2.68, -0.02)


def base(nx: int, ny: int, nz: int, dz: float, dtg: float) -> GwConfig:
    """``gwBaseConfig`` (test_gw.cpp:86-109)."""
    return GwConfig(
        domain=Domain(nx=nx, ny=ny, nz=nz, dx=1.0, dy=1.0, dz=dz, bottom_elevation=0.0),
        soil_types=[test_soil()],
        groundwater=Groundwater(timestep=Timestep(dt_init=dtg, dt_min=dtg, dt_max=dtg),
                                specific_storage=0.0),
        initial=InitialCondition("moisture", 0.2),
        solver=Solver(),
    )


def top_bc(kind: str, value: float, nx: int, ny: int, form: str = "constant") -> BoundaryCondition:
    return BoundaryCondition("top", whole_footprint(nx, ny), "groundwater_top", kind, form, value)


def bottom_bc(kind: str, value: float, nx: int, ny: int, form: str = "constant"):
    return BoundaryCondition("bottom", whole_footprint(nx, ny), "groundwater_bottom", kind, form,
                             value)


WEST_MIDDLE = [(-0.1, 1.1), (0.9, 1.1), (0.9, 1.9), (-0.1, 1.9)]


# ------------------------------------------------------------------ scenarios
def closed_column(ss: float = 0.0) -> GwConfig:
    cfg = base(1, 1, 20, 0.05, 0.5)
    cfg.groundwater.specific_storage = ss
    return cfg


def head_top() -> GwConfig:
    cfg = base(1, 1, 10, 0.05, 0.5)
    cfg.initial = InitialCondition("moisture", 0.06)
    cfg.boundary_conditions = [top_bc("head", 0.0, 1, 1)]
    return cfg


def flux_top() -> GwConfig:
    cfg = base(1, 1, 10, 0.1, 0.5)
    cfg.boundary_conditions = [top_bc("flux", -1.0e-6, 1, 1)]
    return cfg


def gravity_bottom() -> GwConfig:
    cfg = base(1, 1, 10, 0.1, 0.5)
    cfg.groundwater.specific_storage = 1.0e-5
    cfg.initial = InitialCondition("water_table", 0.0)
    cfg.boundary_conditions = [bottom_bc("flux", 0.0, 1, 1, form="gravity")]
    return cfg


def flux_bottom() -> GwConfig:
    cfg = base(1, 1, 10, 0.1, 0.5)
    cfg.boundary_conditions = [bottom_bc("flux", 2.0e-6, 1, 1)]
    return cfg


def hydrostatic_side() -> GwConfig:
    cfg = base(3, 3, 10, 0.1, 0.5)
    cfg.initial = InitialCondition("water_table", -0.35)
    cfg.boundary_conditions = [BoundaryCondition(
        "sea", [(-0.1, 1.1), (0.9, 1.1), (0.9, 1.9), (-0.1, 1.9)], "groundwater_side", "head",
        "hydrostatic", hydrostatic_eta=-0.35)]
    return cfg


def side_flux() -> GwConfig:
    cfg = base(3, 3, 5, 0.1, 0.5)
    cfg.boundary_conditions = [BoundaryCondition("inflow", WEST_MIDDLE, "groundwater_side",
                                                 "flux", "constant", 4.0e-6)]
    return cfg


def full3d(flag: bool) -> GwConfig:
    cfg = base(2, 1, 4, 0.1, 0.5)
    cfg.groundwater.use_full3d = flag
    cfg.initial = InitialCondition(
        "moisture", np.array([0.10, 0.10, 0.10, 0.10, 0.30, 0.30, 0.30, 0.30]).reshape(1, 2, 4))
    return cfg


def sand_over_clay(redistribute: bool = False, off: bool = False,
                   pc: str = "legacy") -> GwConfig:
    cfg = base(1, 1, 10, 0.05, 0.5)
    cfg.groundwater.reallocation = "disabled" if off else "legacy"
    cfg.groundwater.predictor_corrector = pc
    cfg.groundwater.reallocation_surplus = "redistribute" if redistribute else "drop"
    sand = test_soil(3.0e-4, "sand")
    clay = SoilType("clay", 1.52e-6, 1.52e-6, 1.52e-6, 0.4686, 0.106, 1.04, 1.395, 0.0)
    cfg.soil_types = [sand, clay]
    cfg.soil_map = np.array([0, 0, 0, 1, 1, 1, 1, 1, 1, 1]).reshape(1, 1, 10)
    cfg.initial = InitialCondition("moisture", 0.14)
    cfg.boundary_conditions = [top_bc("head", 0.0, 1, 1)]
    return cfg


def adaptive_column() -> GwConfig:
    cfg = base(1, 1, 8, 0.1, 0.1)
    cfg.groundwater.timestep = Timestep(dt_init=0.1, dt_min=0.1, dt_max=1.0)
    cfg.groundwater.specific_storage = 1.0e-5
    cfg.initial = InitialCondition("water_table", 0.0)
    return cfg


def masked_column(gj: int, gi: int) -> GwConfig:
    cfg = base(3, 3, 4, 0.05, 0.5)
    bath = np.zeros((3, 3))
    bath[gj, gi] = -1.0
    cfg.domain.bottom_elevation = bath
    return cfg


def heterogeneous_stack(harmonic: bool, pc: str = "consistent") -> GwConfig:
    cfg = base(1, 1, 6, 0.25, 10.0)
    cfg.groundwater.reallocation = "legacy"
    cfg.groundwater.predictor_corrector = pc
    cfg.groundwater.face_conductivity = "harmonic" if harmonic else "arithmetic"
    cfg.soil_types = [test_soil(math.pow(10.0, -6.5 + 0.6 * n), f"k{n}") for n in range(6)]
    cfg.soil_map = np.array([0, 3, 1, 4, 2, 5]).reshape(1, 1, 6)
    cfg.initial = InitialCondition("water_table", 5.0)
    cfg.boundary_conditions = [top_bc("head", 2.0, 1, 1), bottom_bc("head", 3.3, 1, 1)]
    return cfg


def homogeneous_pair(pc: str) -> GwConfig:
    cfg = base(2, 1, 4, 0.25, 10.0)
    cfg.groundwater.reallocation = "legacy"
    cfg.groundwater.predictor_corrector = pc
    cfg.initial = InitialCondition("moisture", 0.2)
    cfg.boundary_conditions = [top_bc("head", 0.1, 2, 1)]
    return cfg


def ponded_top(pc: str) -> GwConfig:
    cfg = base(1, 1, 6, 0.2, 5.0)
    cfg.groundwater.reallocation = "legacy"
    cfg.groundwater.predictor_corrector = pc
    cfg.initial = InitialCondition("moisture", 0.15)
    cfg.boundary_conditions = [top_bc("head", 0.3, 1, 1)]
    return cfg


def regular_partial_cells() -> GwConfig:
    cfg = base(3, 1, 3, 0.1, 0.5)
    cfg.domain.bottom_elevation = np.array([[0.0, -0.05, -0.09]])
    return cfg


def terrain(uniform: bool) -> GwConfig:
    cfg = base(2, 1, 4, 0.1, 0.5)
    cfg.domain.follow_terrain = True
    cfg.domain.terrain_layers = "uniform" if uniform else "scaled"
    cfg.domain.bottom_elevation = np.array([[0.0, -0.1]])
    return cfg


def mixed_box(seed: int = 7, nx: int = 6, ny: int = 5, nz: int = 12) -> GwConfig:
    """A small 3D box exercising every boundary kind at once: ponded head on
    part of the top, flux elsewhere, head/flux/hydrostatic sides, a masked
    column and partial cells from a rough bed, two soils, Ss > 0."""
    rng = np.random.default_rng(seed)
    cfg = base(nx, ny, nz, 0.05, 2.0)
    cfg.groundwater.timestep = Timestep(dt_init=2.0, dt_min=0.01, dt_max=60.0)
    cfg.groundwater.specific_storage = 1.0e-5
    cfg.groundwater.reallocation_surplus = "redistribute"
    bath = rng.uniform(-0.12, 0.0, size=(ny, nx))
    bath[ny - 1, nx - 1] = -2.0  # fully masked column
    cfg.domain.bottom_elevation = bath
    cfg.soil_types = [test_soil(2e-5, "a"), SoilType("b", 5e-6, 5e-6, 2e-6, 0.42, 0.06, 2.0,
                                                      1.8, 0.0)]
    cfg.soil_map = rng.integers(0, 2, size=(ny, nx, nz))
    cfg.initial = InitialCondition("head", rng.uniform(-1.5, -0.2, size=(ny, nx, nz)))
    half = [(-0.1, -0.1), (nx / 2 + 0.01, -0.1), (nx / 2 + 0.01, ny + 0.1), (-0.1, ny + 0.1)]
    other = [(nx / 2 + 0.01, -0.1), (nx + 0.1, -0.1), (nx + 0.1, ny + 0.1),
             (nx / 2 + 0.01, ny + 0.1)]
    cfg.boundary_conditions = [
        BoundaryCondition("pond", half, "groundwater_top", "head", "constant", 0.02),
        BoundaryCondition("rain", other, "groundwater_top", "flux", "constant", -2e-6),
        BoundaryCondition("drain", whole_footprint(nx, ny), "groundwater_bottom", "flux",
                          "gravity"),
        BoundaryCondition("west", [(-0.1, -0.1), (0.6, -0.1), (0.6, ny + 0.1), (-0.1, ny + 0.1)],
                          "groundwater_side", "head", "hydrostatic", hydrostatic_eta=-0.3),
        BoundaryCondition("south", [(1.1, -0.1), (nx - 1.1, -0.1), (nx - 1.1, 0.6), (1.1, 0.6)],
                          "groundwater_side", "flux", "constant", 1e-6),
        BoundaryCondition("east", [(nx - 0.6, -0.1), (nx + 0.1, -0.1), (nx + 0.1, 2.5),
                                   (nx - 0.6, 2.5)], "groundwater_side", "head", "constant",
                          -0.4),
    ]
    return cfg


def coupled_box(pc: str = "consistent", seed: int = 11, nx: int = 7, ny: int = 6,
                nz: int = 12) -> GwConfig:
    """A small box for the coupled top: rough bed, two soils, Ss > 0, a head
    IC that is saturated (positive, pressurized) in some columns, at the
    retention curve's air-entry value near the top of others and dry
    elsewhere; top flux conditions (infiltration on one half, evaporation on
    a strip), a pushing head at part of the bottom, a hydrostatic west edge
    whose stage stands above the bed, a masked column."""
    rng = np.random.default_rng(seed)
    cfg = base(nx, ny, nz, 0.05, 2.0)
    cfg.groundwater.timestep = Timestep(dt_init=2.0, dt_min=0.01, dt_max=60.0)
    cfg.groundwater.specific_storage = 1.0e-5
    cfg.groundwater.predictor_corrector = pc
    cfg.groundwater.reallocation_surplus = "redistribute"
    bath = rng.uniform(-0.12, 0.0, size=(ny, nx))
    bath[ny - 1, nx - 1] = -2.0  # fully masked column
    cfg.domain.bottom_elevation = bath
    cfg.soil_types = [test_soil(2e-5, "a"), SoilType("b", 5e-6, 5e-6, 2e-6, 0.42, 0.06, 2.0,
                                                      1.8, 0.0)]
    cfg.soil_map = rng.integers(0, 2, size=(ny, nx, nz))
    head = rng.uniform(-1.2, -0.3, size=(ny, nx, nz))
    z = (np.arange(nz) + 0.5) * 0.05
    head[0:2, 0:3, :] = 0.15 + z                 # pressurized, saturated columns
    head[2:4, 3:5, 0:3] = -0.01                  # wet top cells (h above the air-entry value)
    cfg.initial = InitialCondition("head", head)
    half = [(-0.1, -0.1), (nx / 2 + 0.01, -0.1), (nx / 2 + 0.01, ny + 0.1), (-0.1, ny + 0.1)]
    strip = [(nx / 2 + 0.01, -0.1), (nx + 0.1, -0.1), (nx + 0.1, 1.5), (nx / 2 + 0.01, 1.5)]
    cfg.boundary_conditions = [
        BoundaryCondition("rain", half, "groundwater_top", "flux", "constant", -3e-6),
        BoundaryCondition("evap", strip, "groundwater_top", "flux", "constant", 2e-7),
        BoundaryCondition("push", [(-0.1, -0.1), (3.1, -0.1), (3.1, 2.1), (-0.1, 2.1)],
                          "groundwater_bottom", "head", "constant", 0.9),
        BoundaryCondition("drain", [(3.1, 2.1), (nx + 0.1, 2.1), (nx + 0.1, ny + 0.1),
                                    (3.1, ny + 0.1)], "groundwater_bottom", "flux", "gravity"),
        BoundaryCondition("west", [(-0.1, -0.1), (0.6, -0.1), (0.6, ny + 0.1), (-0.1, ny + 0.1)],
                          "groundwater_side", "head", "hydrostatic", hydrostatic_eta=0.04),
    ]
    return cfg


def coupled_surface(bath_halo: np.ndarray, seed: int = 5):
    """Initial free surface and rain rate of the stand-in surface over a
    coupled box: ponds of 5 cm, 1.2 mm (a thin supply-limited film) and
    0.4 mm (below a 1 mm min_depth) on some columns, rain on a block."""
    rng = np.random.default_rng(seed)
    ny2, nx2 = bath_halo.shape
    pond = np.zeros((ny2, nx2))
    pond[3:5, 1:3] = 0.05
    pond[5, 4:6] = 0.0012
    pond[1, 5] = 0.0004
    rain = np.zeros((ny2, nx2))
    rain[4:7, 3:7] = rng.uniform(1e-6, 4e-6, size=rain[4:7, 3:7].shape)
    return bath_halo + pond, rain


def density_scalars(nx: int, ny: int, nz: int, step: int = 0, seed: int = 3):
    """Seeded salinity [g/L] and temperature [C] in the halo layouts
    ((ny+2, nx+2, nz) cells, ghosts included, and (ny+2, nx+2) surfaces), as
    a transport module would hand them over after its step `step`: a saline
    wedge rising toward +x with noise, a warm top layer, both drifting with
    the step so that each step's ratios differ."""
    rng = np.random.default_rng(seed)
    j, i, k = np.meshgrid(np.arange(ny + 2), np.arange(nx + 2), np.arange(nz), indexing="ij")
    wedge = 35.0 * np.clip((i / (nx + 1)) + (k / max(nz - 1, 1)) - 0.6 + 0.05 * step, 0.0, 1.0)
    salt = wedge + 2.0 * rng.random((ny + 2, nx + 2, nz))
    temp = 12.0 + 10.0 * np.exp(-k / max(nz / 4.0, 1.0)) + 0.3 * step + rng.random((ny + 2, nx + 2, nz))
    salt_surf = 5.0 + 30.0 * rng.random((ny + 2, nx + 2))
    temp_surf = 25.0 + 3.0 * rng.random((ny + 2, nx + 2))
    return salt, salt_surf, temp, temp_surf


SCENARIOS = {
    "closed_column": lambda: closed_column(),
    "closed_column_ss": lambda: closed_column(1.0e-4),
    "head_top": head_top,
    "flux_top": flux_top,
    "gravity_bottom": gravity_bottom,
    "flux_bottom": flux_bottom,
    "hydrostatic_side": hydrostatic_side,
    "side_flux": side_flux,
    "full3d_off": lambda: full3d(False),
    "full3d_on": lambda: full3d(True),
    "sand_clay_drop": lambda: sand_over_clay(False),
    "sand_clay_redistribute": lambda: sand_over_clay(True),
    "sand_clay_off": lambda: sand_over_clay(False, off=True, pc="consistent"),
    "adaptive": adaptive_column,
    "masked_west": lambda: masked_column(1, 0),
    "masked_north": lambda: masked_column(2, 1),
    "stack_arith": lambda: heterogeneous_stack(False),
    "stack_harm": lambda: heterogeneous_stack(True),
    "stack_legacy": lambda: heterogeneous_stack(False, "legacy"),
    "pair_legacy": lambda: homogeneous_pair("legacy"),
    "ponded_consistent": lambda: ponded_top("consistent"),
    "partial_cells": regular_partial_cells,
    "terrain_scaled": lambda: terrain(False),
    "terrain_uniform": lambda: terrain(True),
    "mixed_box": mixed_box,
}
