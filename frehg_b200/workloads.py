"""Seeded synthetic groundwater workloads.

There is no public dataset behind these cases: every input is generated here
from fixed seeds with the shapes, sizes and value distributions of the
workloads the step is measured on.

* :func:`column_32x32x50` — homogeneous 32x32x50 box, dz = 0.02 m, ponded
  head 0.01 m on top, free drainage below, no-flux sides, initial head
  -1 m, dt0 = 10 s adaptive (the reference-CPU-runnable case).
* :func:`hillslope` — terrain-following heterogeneous slab (default
  512x512x128, dz = 0.05 m): 2 % planar slope plus seeded Gaussian bumps,
  lnKs Gaussian random field, per-cell van Genuchten parameters, water
  table 2 m below the surface, top flux 1e-6 m/s downward, dt0 = 60 s.
  Smaller sizes give parity crops of the same construction.
* :func:`ensemble` — many independent homogeneous boxes of uneven size
  (nx, ny ~ U{16..128}, nz ~ U{32..200}), per-member van Genuchten
  parameters, lnKs ~ N(ln 1e-5, 1), initial head ~ U[-3, -0.2] m, ponded
  head or flux 1e-6 m/s on top by a seeded coin, free drainage below.

Choices the case descriptions leave open are fixed here and documented in
the docstrings (dt_min / dt_max, bottom condition, theta_s / theta_r / Ss of
the slab, slope axis, bump count).
"""
from __future__ import annotations

import numpy as np

from .config import (BoundaryCondition, Domain, Groundwater, GwConfig, InitialCondition,
                     Solver, SoilType, Timestep, whole_footprint)


def column_32x32x50(nx: int = 32, ny: int = 32, nz: int = 50, precision: str = "fp64",
                    dt_max: float = 600.0) -> GwConfig:
    """Homogeneous infiltration box.

    Soil alpha 1.0 1/m, n 2.0, theta_s 0.40, theta_r 0.05, Ks 1e-5 m/s
    (x, y, z), aev 0, Ss 1e-5 1/m.  dt_min = 1e-3 s and dt_max = 600 s (left
    open by the case description).
    """
    soil = SoilType("c1", 1e-5, 1e-5, 1e-5, 0.40, 0.05, 1.0, 2.0, 0.0)
    fp = whole_footprint(nx, ny)
    return GwConfig(
        domain=Domain(nx=nx, ny=ny, nz=nz, dx=1.0, dy=1.0, dz=0.02, bottom_elevation=0.0),
        soil_types=[soil],
        groundwater=Groundwater(timestep=Timestep(dt_init=10.0, dt_min=1e-3, dt_max=dt_max),
                                specific_storage=1e-5),
        initial=InitialCondition("head", -1.0),
        solver=Solver(precision=precision),
        boundary_conditions=[
            BoundaryCondition("ponded-top", fp, "groundwater_top", "head", "constant", 0.01),
            BoundaryCondition("free-drainage", fp, "groundwater_bottom", "flux", "gravity"),
        ],
    )


def _gaussian_field(shape, corr_cells: float, rng: np.random.Generator) -> np.ndarray:
    """Zero-mean, unit-variance Gaussian random field with a Gaussian
    covariance of correlation length ``corr_cells`` (FFT filter of white
    noise)."""
    noise = rng.standard_normal(shape)
    spec = np.fft.rfftn(noise)
    freqs = [np.fft.fftfreq(n) for n in shape[:-1]] + [np.fft.rfftfreq(shape[-1])]
    grids = np.meshgrid(*freqs, indexing="ij")
    k2 = sum(g * g for g in grids)
    filt = np.exp(-0.5 * (2.0 * np.pi) ** 2 * k2 * corr_cells ** 2 / 2.0)
    field = np.fft.irfftn(spec * filt, s=shape, axes=tuple(range(len(shape))))
    field -= field.mean()
    std = field.std()
    return field / std if std > 0 else field


def hillslope(nx: int = 512, ny: int = 512, nz: int = 128, seed: int = 20261203,
              precision: str = "fp64", n_bumps: int = 64, per_cell_soil: bool = True) -> GwConfig:
    """Terrain-following heterogeneous slab.

    Bed = -0.02 * x (slope along +x) + sum of ``n_bumps`` seeded Gaussian
    bumps (amplitude 0.5 m, sigma 16 cells).  lnKs ~ GRF(mean ln 1e-5,
    sigma 1, correlation 8 cells), Ksx = Ksy = Ksz; alpha ~ U[0.5, 3],
    n ~ U[1.4, 2.5] per cell; theta_s 0.40, theta_r 0.05, aev 0, Ss 1e-5
    (open in the case description; taken from the homogeneous box).
    terrain_layers uniform (the scaled rule rejects relief deeper than the
    slab).  Initial water table 2 m below each column's surface.  Top flux
    -1e-6 m/s (downward, the reference's sign), free-drainage bottom (open
    in the description), no-flux sides.  dt0 = 60 s, dt_min = 1e-3 s,
    dt_max = 600 s.  The head solve gets max_iterations = 20000: the
    Jacobi-preconditioned CG needs more than the reference's default 1000
    iterations on the first 60 s step of every crop from 32x32x128 up (the
    reference treats that as fatal), and several hundred per step after the
    controller's first cut.
    """
    rng = np.random.default_rng(seed)
    dx = dy = 1.0
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dy
    X, Y = np.meshgrid(x, y)  # (ny, nx)
    bath = -0.02 * X
    sigma = 16.0 * dx
    for _ in range(n_bumps):
        cx, cy = rng.uniform(0, nx * dx), rng.uniform(0, ny * dy)
        bath += 0.5 * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2.0 * sigma ** 2))
    ln_ks = np.log(1e-5) + 1.0 * _gaussian_field((ny, nx, nz), 8.0, rng)
    ks = np.exp(ln_ks)
    alpha = rng.uniform(0.5, 3.0, size=(ny, nx, nz))
    vgn = rng.uniform(1.4, 2.5, size=(ny, nx, nz))
    if per_cell_soil:
        types = [SoilType("s", 0, 0, 0, 0.40, 0.05, 0, 0, 0.0)]
        cfg_soil = dict(ksx=ks, ksy=ks, ksz=ks, vg_alpha=alpha, vg_n=vgn)
        soil_map = None
    else:
        types = [SoilType(f"s{n}", k, k, k, 0.40, 0.05, a, m, 0.0)
                 for n, (k, a, m) in enumerate(zip(ks.ravel(), alpha.ravel(), vgn.ravel()))]
        cfg_soil = None
        soil_map = np.arange(nx * ny * nz).reshape(ny, nx, nz)
    fp = whole_footprint(nx, ny, dx, dy)
    cfg = GwConfig(
        domain=Domain(nx=nx, ny=ny, nz=nz, dx=dx, dy=dy, dz=0.05, bottom_elevation=bath,
                      follow_terrain=True, terrain_layers="uniform"),
        soil_types=types,
        groundwater=Groundwater(timestep=Timestep(dt_init=60.0, dt_min=1e-3, dt_max=600.0),
                                specific_storage=1e-5),
        initial=InitialCondition("water_table", bath - 2.0),
        solver=Solver(precision=precision, max_iterations=20000),
        boundary_conditions=[
            BoundaryCondition("recharge", fp, "groundwater_top", "flux", "constant", -1e-6),
            BoundaryCondition("free-drainage", fp, "groundwater_bottom", "flux", "gravity"),
        ],
        soil_map=soil_map,
        cell_soil=cfg_soil,
    )
    return cfg


def ensemble_member(rng: np.random.Generator, precision: str = "fp64",
                    nx_range=(16, 128), nz_range=(32, 200)) -> GwConfig:
    """One member of :func:`ensemble` drawn from ``rng``.

    Sizes nx, ny ~ U{16..128}, nz ~ U{32..200}; dx = dy = 1 m, dz = 0.02 m
    (the box case's grid).  Soil: alpha ~ U[0.5, 3] 1/m, n ~ U[1.4, 2.5],
    theta_s = 0.40, theta_r = 0.05 (the box case's), lnKs ~ N(ln 1e-5, 1)
    with Ksx = Ksy = Ksz, Ss = 1e-5 1/m.  Initial head uniform in the member,
    drawn from U[-3, -0.2] m.  Top: ponded head 0.01 m or flux 1e-6 m/s
    downward by a fair coin; bottom free drainage; sides no-flux.  dt0 = 10 s,
    dt_min = 1e-3 s, dt_max = 600 s.
    """
    nx = int(rng.integers(nx_range[0], nx_range[1] + 1))
    ny = int(rng.integers(nx_range[0], nx_range[1] + 1))
    nz = int(rng.integers(nz_range[0], nz_range[1] + 1))
    ks = float(np.exp(np.log(1e-5) + rng.standard_normal()))
    alpha = float(rng.uniform(0.5, 3.0))
    vgn = float(rng.uniform(1.4, 2.5))
    h0 = float(rng.uniform(-3.0, -0.2))
    ponded = bool(rng.integers(0, 2))
    soil = SoilType("member", ks, ks, ks, 0.40, 0.05, alpha, vgn, 0.0)
    fp = whole_footprint(nx, ny)
    top = (BoundaryCondition("ponded-top", fp, "groundwater_top", "head", "constant", 0.01)
           if ponded else
           BoundaryCondition("recharge-top", fp, "groundwater_top", "flux", "constant", -1e-6))
    return GwConfig(
        domain=Domain(nx=nx, ny=ny, nz=nz, dx=1.0, dy=1.0, dz=0.02, bottom_elevation=0.0),
        soil_types=[soil],
        groundwater=Groundwater(timestep=Timestep(dt_init=10.0, dt_min=1e-3, dt_max=600.0),
                                specific_storage=1e-5),
        initial=InitialCondition("head", h0),
        solver=Solver(precision=precision),
        boundary_conditions=[
            top,
            BoundaryCondition("free-drainage", fp, "groundwater_bottom", "flux", "gravity"),
        ],
    )


def ensemble(n: int = 256, seed: int = 20261204, precision: str = "fp64",
             nx_range=(16, 128), nz_range=(32, 200)) -> list:
    """``n`` independent members (see :func:`ensemble_member`), seeded."""
    rng = np.random.default_rng(seed)
    return [ensemble_member(rng, precision, nx_range, nz_range) for _ in range(n)]
