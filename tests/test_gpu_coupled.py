"""The coupled top and the coupler window on the B200 against the oracle.

The oracle's coupled branches and coupler are pinned bit for bit to the
reference's own sources (tests/test_oracle_coupled.py); here the CUDA path
(through the C ABI) must follow them on the same coupled box with the bars
of the groundwater-only step.  FP64 form, in lockstep with the default
oracle: head within 1e-9 relative L-inf, other fields and the surface fields
within 1e-8 of their scale, the same exchange mode in every column, CG
iterations within +-2, the coupled audit terms within 1e-9 of their scale.
Mixed form, against the FP64 oracle solved tightly (rtol 1e-13) from the
GPU's state each step (window): head within 1e-8, the surface fields and
audit terms within 1e-6 (fluxes carry the head error over half a cell).
Both: the GPU's own per-step mass audit closes to 1e-12 of the storage.
"""
import copy

import numpy as np
import pytest

import cases
from frehg_b200.batch import RichardsBatch
from frehg_b200.coupling import Coupler
from frehg_b200.gw import FatalError, RichardsSolver
from oracle.gw import OracleSolver

pytestmark = pytest.mark.gpu

MIN_DEPTH = 0.001
# Volume scale of the audit comparisons [m^3]: a term smaller than this (the
# box holds ~10 m^3 of water) is compared absolutely against it.
VOL_FLOOR = 1e-6
SURF = ("eta", "dept", "seep_accum", "avail", "gain")


def rel(a, b, floor=1e-12):
    scale = max(float(np.max(np.abs(b))), floor)
    return float(np.max(np.abs(a - b)) / scale)


def refresh_depth(eta, bottom):
    d = eta - bottom
    d[d <= MIN_DEPTH] = 0.0
    return d


def htol(cfg):
    return 1e-8 if cfg.solver.precision == "mixed" else 1e-9


def ftol(cfg):
    return 1e-6 if cfg.solver.precision == "mixed" else 1e-8


def check_fields(g, o, cfg, tag):
    assert rel(g.field("h"), o.field("h"), 1.0) <= htol(cfg), tag
    for name in ("wc", "qx", "qy", "qz", "kz"):
        assert rel(g.field(name), o.field(name)) <= ftol(cfg), f"{name} {tag}"


def oracle_for(cfg):
    """The default oracle for the FP64 form; for the mixed form the FP64
    oracle with a tight solve (it is re-synced to the GPU's state)."""
    c = copy.deepcopy(cfg)
    if cfg.solver.precision == "mixed":
        c.solver.precision = "fp64"
        c.solver.rtol = 1e-13
        c.solver.atol = 1e-300
        c.solver.max_iterations = 200000
    return OracleSolver(c)


def sync_oracle(o, g, names):
    o.set_state(g.head(), g.waterContent())
    for name in names:
        o.set_surface(name, g.surface(name))


@pytest.mark.parametrize("pc,precision,vent_all,bounce", [
    ("consistent", "fp64", False, False),
    ("legacy", "fp64", False, True),
    ("consistent", "mixed", True, True),
])
def test_coupled_steps_match_oracle(pc, precision, vent_all, bounce):
    cfg = cases.coupled_box(pc)
    cfg.solver.precision = precision
    mixed = precision == "mixed"
    o = oracle_for(cfg)
    g = RichardsSolver(copy.deepcopy(cfg))
    names = SURF + (("bounce",) if bounce else ())
    try:
        o.attach_coupling(MIN_DEPTH, vent_all, bounce)
        g.attachCoupling(MIN_DEPTH, vent_all, bounce)
        bath = o.bath_halo()
        eta, _ = cases.coupled_surface(bath)
        d = refresh_depth(eta, bath)
        for name, v in (("eta", eta), ("dept", d), ("avail", d)):
            o.set_surface(name, v)
            g.setSurface(name, v)
        prev = g.ownedVolume()
        t = 0.0
        for n in range(10):
            if mixed:
                sync_oracle(o, g, names)
                dtg = g.nextDt()
            else:
                dtg = o.next_dt()
                assert g.nextDt() == pytest.approx(dtg, rel=1e-9), n
            t += dtg
            o.step(t, dtg)
            info = g.step(t, dtg)
            if not mixed:  # the mixed form's inner iterations are its own
                assert abs(info["cg_iterations"] - o.info["cg_iterations"]) <= 2, n
            np.testing.assert_array_equal(g.surface("mode"), o.surface("mode"), err_msg=f"{n}")
            check_fields(g, o, cfg, f"step {n}")
            for name in names:
                assert rel(g.surface(name), o.surface(name)) <= ftol(cfg), f"{name} step {n}"
            ga, oa = g.couplingAudit(), o.coupled_audit()
            atol = 1e-6 if mixed else 1e-9
            for k, v in oa.items():
                if k == "pc_clamp_volume" and mixed:
                    continue  # cumulative: the oracle's restarts each step
                assert abs(ga[k] - v) <= atol * max(abs(v), VOL_FLOOR), f"{k} step {n}"
            v = g.ownedVolume()
            resid = (v - prev) - (info["boundary_in"] - info["ss_storage"] +
                                  info["realloc_adjust"] - info["vloss"])
            assert abs(resid) <= 1e-12 * max(v, 1.0), (n, resid)
            prev = v
        assert g.couplingAudit()["vent"] > 0.0
    finally:
        g.close()
        o.close()


@pytest.mark.parametrize("sync,precision", [(True, "fp64"), (False, "fp64"), (False, "mixed")])
def test_coupler_windows_match_oracle(sync, precision):
    cfg = cases.coupled_box("consistent")
    cfg.solver.precision = precision
    mixed = precision == "mixed"
    o = oracle_for(cfg)
    g = RichardsSolver(copy.deepcopy(cfg))
    try:
        dt = 5.0
        o.attach_coupling(MIN_DEPTH)
        o.coupler_init(sync, dt, 2.0, 0.0)
        g.attachCoupling(MIN_DEPTH)
        cp = Coupler(g, sync, dt, 2.0, 0.0)
        bath = o.bath_halo()
        eta, rain = cases.coupled_surface(bath)
        o.set_surface("eta", eta)
        g.setSurface("eta", eta)
        g.setSurface("bottom", bath)
        t = 0.0
        tol = 1e-6 if mixed else 1e-9
        for n in range(8):
            if mixed:
                sync_oracle(o, g, ("eta", "seep_accum"))
                o.coupler_restore(t, cp.currentDtg(), cp.gwLag(t))
            step_dt = o.coupler_state(t)[0]
            assert cp.nextDt() == pytest.approx(step_dt, rel=1e-9), n
            t += step_dt
            for x, get, put in ((o, o.surface, o.set_surface), (g, g.surface, g.setSurface)):
                e = get("eta") + rain * step_dt
                put("eta", e)
                put("dept", refresh_depth(e, bath))
            wo = o.coupler_step(t, step_dt, bath)
            wg = cp.step(t, step_dt)
            assert wg["substeps"] == wo["substeps"], n
            for k in ("boundary_in", "ss_storage", "realloc_adjust", "vloss"):
                assert abs(wg["gw"][k] - wo["gw"][k]) <= tol * max(abs(wo["gw"][k]), VOL_FLOOR), k
            for k in ("exchanged", "bounce", "vent", "evap"):
                assert abs(wg["cpl"][k] - wo["cpl"][k]) <= tol * max(abs(wo["cpl"][k]), VOL_FLOOR), k
            for k in ("applied", "discarded", "surface_gain", "accum_volume"):
                assert abs(wg[k] - wo[k]) <= tol * max(abs(wo[k]), VOL_FLOOR), (k, n)
            check_fields(g, o, cfg, f"window {n}")
            for name in ("eta", "dept", "seep_accum", "gain", "qss"):
                assert rel(g.surface(name), o.surface(name)) <= ftol(cfg), f"{name} window {n}"
        assert cp.gwLag(t) == pytest.approx(o.coupler_state(t)[2], abs=1e-9)
    finally:
        g.close()
        o.close()


def test_batch_refuses_coupled_members():
    cfg = cases.coupled_box()
    a = RichardsSolver(copy.deepcopy(cfg))
    b = RichardsSolver(copy.deepcopy(cfg))
    try:
        a.attachCoupling(MIN_DEPTH)
        with pytest.raises(FatalError):
            RichardsBatch([a, b])
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("sync", [True, False])
def test_coupled_budget_closes(sync):
    # The coupled closure (Coupler.hpp:51-57) with the stand-in surface's
    # rain as the surface source: d(V_gw + V_surface + held seepage) = rain +
    # the external boundary inflow (boundary_in + exchanged + vent) + bounce
    # - evaporation - Ss storage + reallocation - clamp loss + the
    # infiltration remainder the bed clamp kept from the surface.
    cfg = cases.coupled_box("consistent")
    g = RichardsSolver(copy.deepcopy(cfg))
    o = OracleSolver(copy.deepcopy(cfg))
    try:
        g.attachCoupling(MIN_DEPTH)
        cp = Coupler(g, sync, 5.0, 2.0)
        bath = o.bath_halo()
        eta, rain = cases.coupled_surface(bath)
        g.setSurface("eta", eta)
        g.setSurface("bottom", bath)

        def surface_volume():
            e, a = g.surface("eta"), g.surface("seep_accum")
            return float(np.sum((e - bath)[1:-1, 1:-1]) + np.sum(a[1:-1, 1:-1]))

        total = g.ownedVolume() + surface_volume()
        t = 0.0
        for n in range(10):
            dt = cp.nextDt()
            t += dt
            e = g.surface("eta") + rain * dt
            g.setSurface("eta", e)
            g.setSurface("dept", refresh_depth(e, bath))
            total += float(np.sum((rain * dt)[1:-1, 1:-1]))
            a = cp.step(t, dt)
            now = g.ownedVolume() + surface_volume()
            src = ((a["gw"]["boundary_in"] + a["cpl"]["exchanged"] + a["cpl"]["vent"]) +
                   a["cpl"]["bounce"] - a["cpl"]["evap"] - a["gw"]["ss_storage"] +
                   a["gw"]["realloc_adjust"] - a["gw"]["vloss"] + a["discarded"])
            assert abs((now - total) - src) <= 1e-12 * max(now, 1.0), (n, now - total, src)
            total = now
    finally:
        g.close()
        o.close()
