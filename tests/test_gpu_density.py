"""Density coupling on the B200 against the oracle.

The oracle's density coupling is pinned bit for bit to the reference's own
sources (tests/test_oracle_density.py); here the CUDA path (through the C
ABI) must follow it with the bars of the groundwater-only step while a
salinity and a temperature are handed over before every step: the cell and
face ratios within 1e-14 of 1 (the same formulas, contraction aside), and in
the FP64 form head within 1e-9 relative L-inf, the other fields within 1e-8
of their scale (fluxes on the gravity scale), CG iterations within +-2 and
the next dt within 1e-9.  The mixed form is compared against the FP64 oracle
solved tightly (rtol 1e-13) from the GPU's state each step: head within
1e-8, fields within 1e-6, with the outer target at 1e-12 (on the small
hydrostatic-side column a residual of 1e-11 left the head 1.2e-8 from the
tight solve: the column's conditioning, not the coupling).  The audit terms follow the oracle's (1e-9 / 1e-6
of their scale).  The volume audit of the groundwater-only step does not
close under density coupling (the theta update conserves r-weighted mass,
face by face): in the FP64 form the GPU's closure residual must equal the
oracle's to 1e-12 of the storage instead.
"""
import copy

import numpy as np
import pytest

import cases
from frehg_b200.batch import RichardsBatch
from frehg_b200.gw import FatalError, RichardsSolver
from oracle.gw import OracleSolver

pytestmark = pytest.mark.gpu

RATIOS = ("rho", "visc", "rho_x", "rho_y", "rho_z", "visc_x", "visc_y", "visc_z")
FLUX_SCALE = {"qx": ("kx", "ax"), "qy": ("ky", "ay"), "qz": ("kz", None)}
MIN_DEPTH = 0.001
VOL_FLOOR = 1e-6  # audit terms below this volume [m^3] are compared against it
AUDIT = ("boundary_in", "ss_storage", "realloc_adjust", "realloc_dropped", "vloss")
DENSITY = {
    "saline": dict(saline=True),
    "both_gradient": dict(saline=True, thermal=True, thermal_expansion=2.0e-4,
                          reallocation_gradient=True),
}


def rel(a, b, floor):
    scale = max(float(np.max(np.abs(b))), floor)
    return float(np.max(np.abs(a - b)) / scale)


def oracle_for(cfg, mixed):
    c = copy.deepcopy(cfg)
    if mixed:
        c.solver.precision = "fp64"
        c.solver.rtol = 1e-13
        c.solver.atol = 1e-300
        c.solver.max_iterations = 200000
    return OracleSolver(c)


def hand_over(g, o, cfg, step, kw):
    d = cfg.domain
    salt, salt_surf, temp, temp_surf = cases.density_scalars(d.nx, d.ny, d.nz, step)
    if kw.get("saline", True):
        g.setScalar("salt", salt)
        g.setScalar("salt_surf", salt_surf)
        o.set_scalar("salt", salt)
        o.set_scalar("salt_surf", salt_surf)
    if kw.get("thermal", False):
        g.setScalar("temp", temp)
        g.setScalar("temp_surf", temp_surf)
        o.set_scalar("temp", temp)
        o.set_scalar("temp_surf", temp_surf)


def check(g, o, cfg, info, mixed, tag):
    for name in RATIOS:
        assert float(np.max(np.abs(g.field(name) - o.field(name)))) <= 1e-14, f"{name} {tag}"
    htol, ftol = (1e-8, 1e-6) if mixed else (1e-9, 1e-8)
    assert rel(g.field("h"), o.field("h"), 1.0) <= htol, f"h {tag}"
    for name in ("wc", "qx", "qy", "qz", "kx", "ky", "kz"):
        floor = 1e-12
        if name in FLUX_SCALE:
            kname, area = FLUX_SCALE[name]
            a = cfg.domain.dx * cfg.domain.dy if area is None else o.field(area)
            floor = max(floor, float(np.max(np.abs(o.field(kname)) * a)))
        assert rel(g.field(name), o.field(name), floor) <= ftol, f"{name} {tag}"
    if not mixed:
        assert abs(info["cg_iterations"] - o.info["cg_iterations"]) <= 2, tag


def run(cfg, kw, mixed, steps=6, coupled=False):
    cfg = copy.deepcopy(cfg)
    cfg.solver.precision = "mixed" if mixed else "fp64"
    if mixed:
        cfg.solver.outer_rtol = 1e-12
    g = RichardsSolver(copy.deepcopy(cfg))
    o = oracle_for(cfg, mixed)
    try:
        if coupled:
            g.attachCoupling(MIN_DEPTH)
            o.attach_coupling(MIN_DEPTH)
            bath = o.bath_halo()
            eta, _ = cases.coupled_surface(bath)
            d = eta - bath
            d[d <= MIN_DEPTH] = 0.0
            for name, v in (("eta", eta), ("dept", d), ("avail", d)):
                g.setSurface(name, v)
                o.set_surface(name, v)
        g.attachDensity(**kw)
        o.attach_density(**kw)
        prev, oprev = g.ownedVolume(), o.owned_volume()
        t = 0.0
        for n in range(steps):
            hand_over(g, o, cfg, n, kw)
            if mixed:
                o.set_state(g.head(), g.waterContent())
                if coupled:
                    for name in ("eta", "dept", "avail", "seep_accum", "gain"):
                        o.set_surface(name, g.surface(name))
                dtg = g.nextDt()
            else:
                dtg = o.next_dt()
                assert g.nextDt() == pytest.approx(dtg, rel=1e-9), n
            t += dtg
            o.step(t, dtg)
            info = g.step(t, dtg)
            check(g, o, cfg, info, mixed, f"step {n}")
            atol = 1e-6 if mixed else 1e-9
            for k in AUDIT:
                ov = o.info[k]
                assert abs(info[k] - ov) <= atol * max(abs(ov), VOL_FLOOR), f"{k} step {n}"
            v, ov = g.ownedVolume(), o.owned_volume()
            if not mixed:
                def closure(dv, a):
                    return dv - (a["boundary_in"] - a["ss_storage"] + a["realloc_adjust"] -
                                 a["vloss"])
                rg, ro = closure(v - prev, info), closure(ov - oprev, o.info)
                assert abs(rg - ro) <= 1e-12 * max(v, 1.0), (n, rg, ro)
            prev, oprev = v, ov
        assert float(np.max(np.abs(g.field("rho") - 1.0))) > 1e-4
    finally:
        g.close()
        o.close()


@pytest.mark.parametrize("name", ["hydrostatic_side", "side_flux", "stack_legacy",
                                  "ponded_consistent", "terrain_uniform", "mixed_box"])
@pytest.mark.parametrize("mode", sorted(DENSITY))
def test_density_fp64_matches_oracle(name, mode):
    run(cases.SCENARIOS[name](), DENSITY[mode], mixed=False)


@pytest.mark.parametrize("name", ["hydrostatic_side", "mixed_box"])
def test_density_mixed_matches_oracle(name):
    run(cases.SCENARIOS[name](), DENSITY["both_gradient"], mixed=True)


@pytest.mark.parametrize("mixed", [False, True])
def test_density_coupled_matches_oracle(mixed):
    run(cases.coupled_box("consistent"), DENSITY["both_gradient"], mixed=mixed, steps=8,
        coupled=True)


def test_unattached_ratios_are_one_and_batch_refuses_density():
    cfg = cases.SCENARIOS["mixed_box"]()
    a = RichardsSolver(copy.deepcopy(cfg))
    b = RichardsSolver(copy.deepcopy(cfg))
    try:
        for name in RATIOS:
            assert np.all(a.field(name) == 1.0), name
        a.attachDensity()
        with pytest.raises(FatalError):
            a.attachDensity()  # once only
        with pytest.raises(FatalError):
            RichardsBatch([a, b])
    finally:
        a.close()
        b.close()


def test_density_with_transport_window_matches_oracle():
    # FP64 form in lockstep with the oracle, density coupling and the window
    # both on: the windows within 1e-8 of their scale (floor: the faces'
    # gravity term K A times the elapsed time, as in the window test).
    from frehg_b200.abi import interior_from_halo

    cfg = copy.deepcopy(cases.SCENARIOS["hydrostatic_side"]())
    cfg.solver.precision = "fp64"
    kw = DENSITY["both_gradient"]
    g = RichardsSolver(copy.deepcopy(cfg))
    o = OracleSolver(cfg)
    try:
        g.attachDensity(**kw)
        o.attach_density(**kw)
        g.enableTransportWindow()
        o.enable_transport_window()
        d = cfg.domain
        t = elapsed = 0.0
        names = {"x": "win_x", "y": "win_y", "z": "win_z"}
        for n in range(6):
            hand_over(g, o, cfg, n, kw)
            dtg = o.next_dt()
            t += dtg
            elapsed += dtg
            o.step(t, dtg)
            info = g.step(t, dtg)
            check(g, o, cfg, info, False, f"step {n}")
            floor = {"x": float(np.max(np.abs(g.field("kx") * g.field("ax")))),
                     "y": float(np.max(np.abs(g.field("ky") * g.field("ay")))),
                     "z": float(np.max(np.abs(g.field("kz")))) * d.dx * d.dy}
            for w, name in names.items():
                ref = interior_from_halo(name, o.window(w), d.nx, d.ny, d.nz)
                fl = max(floor[w] * elapsed, 1e-15)
                assert rel(g.field(name), ref, fl) <= 1e-8, f"window {w} step {n}"
    finally:
        g.close()
        o.close()
