"""Pin the oracle's coupled top against the reference's own sources.

The coupled branches of the step (exchange-mode classification, the top
face conductivity, assembly, top flux, bookkeeping, the reallocation's
wet-top contact and surface vent, the hydrostatic edge ghost) and the
reference's ``coupling::Coupler`` window (sync and subcycled, the seepage
application and its audit) run in ``oracle/_ref`` over a stand-in surface
without lateral flow (``oracle/shim/include/swe/SurfaceSolver.hpp``: rain
into eta, the surface solver's depth rule).  The restatement must reproduce
them bit for bit: fields, surface fields, every audit term, CG iterations
and the controllers' dts.
"""
import numpy as np
import pytest

import cases
from oracle import ref as refmod
from oracle.gw import OracleSolver

pytestmark = pytest.mark.skipif(not refmod.available(), reason="oracle/_ref not built")

FIELDS = ("h", "wc", "qx", "qy", "qz", "kx", "ky", "kz")
MIN_DEPTH = 0.001


def refresh_depth(eta, bottom, min_depth=MIN_DEPTH):
    """The stand-in surface's depth rule (src/swe/WetDry.cpp:24-43)."""
    d = eta - bottom
    d[d <= min_depth] = 0.0
    return d


def compare_state(r, o, tag, surf=("eta", "dept", "seep_accum", "gain")):
    for name in FIELDS:
        np.testing.assert_array_equal(o.field(name), r.field(name), err_msg=f"{name} {tag}")
    for name in surf:
        np.testing.assert_array_equal(o.surface(name), r.surface(name), err_msg=f"{name} {tag}")


@pytest.mark.parametrize("pc,vent_all,bounce", [("consistent", False, False),
                                                ("legacy", False, True),
                                                ("consistent", True, True)])
def test_coupled_steps_bitwise(pc, vent_all, bounce):
    cfg = cases.coupled_box(pc)
    r = refmod.RefSolver(cfg, pc="jacobi")
    o = OracleSolver(cfg)
    r.attach_coupling(MIN_DEPTH, vent_all, bounce)
    o.attach_coupling(MIN_DEPTH, vent_all, bounce)
    bath = r.halo_field("bath")
    eta, _ = cases.coupled_surface(bath)
    d = refresh_depth(eta, bath)
    for x in (r, o):
        x.set_surface("eta", eta)
        x.set_surface("dept", d)
        x.set_surface("avail", d)
    seen = set()
    for n in range(10):
        r.advance()
        o.advance()
        its, res = r.last_solve()
        assert o.info["cg_iterations"] == its, n
        assert o.info["residual_norm"] == res, n
        assert o.next_dt() == r.next_dt(), n
        a = r.audit()
        for k in ("boundary_in", "ss_storage", "realloc_adjust", "realloc_dropped", "vloss"):
            assert o.info[k] == a[k], f"{k} step {n}"
        assert o.coupled_audit() == r.coupled_audit(), n
        compare_state(r, o, f"step {n}", ("eta", "dept", "seep_accum", "avail", "gain") +
                      (("bounce",) if bounce else ()))
        seen.update(np.unique(o.surface("mode")[1:-1, 1:-1]).astype(int).tolist())
    # the box exercises every exchange mode its form has
    assert seen == ({0, 1, 2, 3} if pc == "consistent" else {0, 1, 2})
    cpl = o.coupled_audit()
    assert cpl["vent"] > 0.0 and cpl["evap"] > 0.0


@pytest.mark.parametrize("sync", [True, False])
def test_coupler_windows_bitwise(sync):
    cfg = cases.coupled_box("consistent")
    r = refmod.RefSolver(cfg, pc="jacobi")
    o = OracleSolver(cfg)
    dt = 5.0
    r.coupler_create(sync, dt, 2.0, 0.0, MIN_DEPTH)
    o.attach_coupling(MIN_DEPTH)
    o.coupler_init(sync, dt, 2.0, 0.0)
    bath = r.halo_field("bath")
    eta, rain = cases.coupled_surface(bath)
    r.set_surface("bottom", bath)
    r.set_surface("rain", rain)
    r.set_surface("eta", eta)
    o.set_surface("eta", eta)
    t = 0.0
    total_sub = 0
    for n in range(8):
        step_dt = r.coupler_state(t)[0]
        assert o.coupler_state(t)[0] == step_dt
        t += step_dt
        # the surface phase of Coupler::step on the stand-in: rain, then depth
        e = o.surface("eta") + rain * step_dt
        o.set_surface("eta", e)
        o.set_surface("dept", refresh_depth(e, bath))
        wa = r.coupler_step(t, step_dt)
        wo = o.coupler_step(t, step_dt, bath)
        assert wo["substeps"] == wa["substeps"], n
        total_sub += wa["substeps"]
        for k, v in wa["gw"].items():
            assert wo["gw"][k] == v, f"{k} window {n}"
        for k, v in wa["cpl"].items():
            assert wo["cpl"][k] == v, f"{k} window {n}"
        for k in ("applied", "discarded", "surface_gain", "accum_volume"):
            assert wo[k] == wa[k], f"{k} window {n}"
        assert o.coupler_state(t) == r.coupler_state(t), n
        compare_state(r, o, f"window {n}", ("eta", "dept", "seep_accum", "gain", "qss"))
    if sync:
        assert total_sub == 8
    else:
        assert total_sub > 8  # the subsurface subcycles inside the 5 s surface steps
