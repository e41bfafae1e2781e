"""Pin the oracle's density coupling against the reference's own sources.

With a salinity and/or temperature attached (RichardsSolver::attachScalar
with baroclinic on, attachTemperature, setDensityCoefficients) the step
computes the cell and face density / viscosity ratios from the scalars at
its start (Baroclinic.cpp) and carries them through the hydrostatic edge
ghosts, the assembly's legs, gravity, boundary-flux and storage terms, the
Darcy fluxes, the theta update, the coupled top's pressurization test and,
with the density reallocation gradient, the post-allocation split.  The
restatement must reproduce the reference bit for bit: the ratios, the state
and flux fields, the audit terms, CG iterations and the controller's dt, on
scenarios covering head, hydrostatic, flux and gravity edges, both
predictor-corrector forms, terrain and the coupled top.
"""
import numpy as np
import pytest

import cases
from oracle import ref as refmod
from oracle.gw import OracleSolver

pytestmark = pytest.mark.skipif(not refmod.available(), reason="oracle/_ref not built")

FIELDS = ("h", "wc", "qx", "qy", "qz", "kx", "ky", "kz")
RATIOS = ("rho", "visc", "rho_y", "rho_z")  # the reference's public accessors
MIN_DEPTH = 0.001


def hand_over(r, o, cfg, step, saline, thermal):
    d = cfg.domain
    salt, salt_surf, temp, temp_surf = cases.density_scalars(d.nx, d.ny, d.nz, step)
    for x in (r, o):
        if saline:
            x.set_scalar("salt", salt)
            x.set_scalar("salt_surf", salt_surf)
        if thermal:
            x.set_scalar("temp", temp)
            x.set_scalar("temp_surf", temp_surf)


def compare(r, o, tag):
    its, res = r.last_solve()
    assert o.info["cg_iterations"] == its, tag
    assert o.info["residual_norm"] == res, tag
    assert o.next_dt() == r.next_dt(), tag
    a = r.audit()
    for k in ("boundary_in", "ss_storage", "realloc_adjust", "realloc_dropped", "vloss"):
        assert o.info[k] == a[k], f"{k} {tag}"
    for name in FIELDS + RATIOS:
        np.testing.assert_array_equal(o.field(name), r.field(name), err_msg=f"{name} {tag}")


DENSITY = {
    "saline": dict(saline=True),
    "thermal": dict(saline=False, thermal=True, thermal_expansion=2.0e-4),
    "both_gradient": dict(saline=True, thermal=True, thermal_expansion=2.0e-4,
                          reallocation_gradient=True),
}


@pytest.mark.parametrize("name", ["hydrostatic_side", "side_flux", "gravity_bottom",
                                  "head_top", "flux_bottom", "sand_clay_redistribute",
                                  "stack_harm", "stack_legacy", "ponded_consistent",
                                  "terrain_uniform", "mixed_box"])
@pytest.mark.parametrize("mode", sorted(DENSITY))
def test_density_bitwise(name, mode):
    cfg = cases.SCENARIOS[name]()
    r = refmod.RefSolver(cfg, pc="jacobi")
    o = OracleSolver(cfg)
    kw = DENSITY[mode]
    for x in (r, o):
        x.attach_density(**kw)
    for n in range(6):
        hand_over(r, o, cfg, n, kw.get("saline", True), kw.get("thermal", False))
        r.advance()
        o.advance()
        compare(r, o, f"{name} {mode} step {n}")
    rho = o.field("rho")
    assert float(np.max(np.abs(rho - 1.0))) > 1e-4  # the ratios moved off 1


@pytest.mark.parametrize("pc", ["consistent", "legacy"])
def test_density_coupled_bitwise(pc):
    # The face above a coupled column's top cell averages with the surface
    # scalar's ratio; the consistent form's pressurization test scales by r.
    cfg = cases.coupled_box(pc)
    r = refmod.RefSolver(cfg, pc="jacobi")
    o = OracleSolver(cfg)
    for x in (r, o):
        x.attach_coupling(MIN_DEPTH)
        x.attach_density(saline=True, thermal=True, thermal_expansion=2.0e-4,
                         reallocation_gradient=True)
    bath = r.halo_field("bath")
    eta, _ = cases.coupled_surface(bath)
    d = eta - bath
    d[d <= MIN_DEPTH] = 0.0
    for x in (r, o):
        x.set_surface("eta", eta)
        x.set_surface("dept", d)
        x.set_surface("avail", d)
    for n in range(8):
        hand_over(r, o, cfg, n, True, True)
        r.advance()
        o.advance()
        compare(r, o, f"coupled {pc} step {n}")
        assert o.coupled_audit() == r.coupled_audit(), n
        for name in ("eta", "dept", "seep_accum", "avail", "gain"):
            np.testing.assert_array_equal(o.surface(name), r.surface(name), err_msg=name)


def test_unattached_ratios_are_one():
    cfg = cases.SCENARIOS["mixed_box"]()
    o = OracleSolver(cfg)
    o.advance()
    for name in ("rho", "visc", "rho_x", "rho_y", "rho_z", "visc_x", "visc_y", "visc_z"):
        assert np.all(o.field(name) == 1.0), name


def test_density_restart_bitwise():
    # refreshDerivedState (RichardsSolver.cpp:880-890) recomputes the ratios
    # before the ghosts: a state overwritten mid-run then stepped matches.
    cfg = cases.SCENARIOS["hydrostatic_side"]()
    r = refmod.RefSolver(cfg, pc="jacobi")
    o = OracleSolver(cfg)
    kw = DENSITY["both_gradient"]
    for x in (r, o):
        x.attach_density(**kw)
    for n in range(3):
        hand_over(r, o, cfg, n, True, True)
        r.advance()
        o.advance()
    h, wc = o.field("h"), o.field("wc")
    h = h + 0.01 * np.sin(np.arange(h.size)).reshape(h.shape)
    hand_over(r, o, cfg, 7, True, True)
    r.set_state_interior(h, wc)
    o.set_state(h, wc)
    for name in ("h", "rho", "rho_y", "rho_z"):
        np.testing.assert_array_equal(o.field(name), r.field(name), err_msg=name)
    for n in range(3):
        hand_over(r, o, cfg, 8 + n, True, True)
        r.advance()
        o.advance()
        compare(r, o, f"after restart {n}")


def test_density_with_transport_window_bitwise():
    # The window accumulates the step's volumetric face fluxes q dtg and the
    # walks' path records; with the density ratios in the fluxes it must
    # still follow the reference's bit for bit.
    cfg = cases.SCENARIOS["hydrostatic_side"]()
    r = refmod.RefSolver(cfg, pc="jacobi")
    o = OracleSolver(cfg)
    kw = DENSITY["both_gradient"]
    for x in (r, o):
        x.attach_density(**kw)
        x.enable_transport_window()
    for n in range(6):
        hand_over(r, o, cfg, n, True, True)
        r.advance()
        o.advance()
        compare(r, o, f"window step {n}")
        for name in ("x", "y", "z"):
            np.testing.assert_array_equal(o.window(name), r.window(name), err_msg=f"{name} {n}")
