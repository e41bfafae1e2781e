"""The transport window on the B200 against the oracle.

The oracle's window (face volumes of every step, the walks' path records on
every crossed face, the vented volumes) is pinned bit for bit to the
reference's own sources (tests/test_oracle_window.py).  Through the C ABI the
CUDA path must follow it in lockstep with the FP64 form: each window within
1e-8 of its own scale (floor 1e-15 m^3), across a reset, on columns whose walks
cross faces beyond their receivers and on a coupled box that vents.
"""
import copy

import numpy as np
import pytest

import cases
from frehg_b200.abi import interior_from_halo
from frehg_b200.batch import RichardsBatch
from frehg_b200.gw import FatalError, RichardsSolver
from oracle.gw import OracleSolver

pytestmark = pytest.mark.gpu

NAMES = {"x": "win_x", "y": "win_y", "z": "win_z", "vent": "win_vent"}


def rel(a, b, floor=1e-15):
    scale = max(float(np.max(np.abs(b))), floor)
    return float(np.max(np.abs(a - b)) / scale)


def check(g, o, cfg, tag, elapsed, vent=False):
    # A window near equilibrium is a cancellation residue of the gravity
    # term K A of its faces (the step parity test's flux scale), so its floor
    # is that scale times the window's elapsed time.
    d = cfg.domain
    floor = {"x": float(np.max(np.abs(g.field("kx") * g.field("ax")))),
             "y": float(np.max(np.abs(g.field("ky") * g.field("ay")))),
             "z": float(np.max(np.abs(g.field("kz")))) * d.dx * d.dy}
    for w in ("x", "y", "z") + (("vent",) if vent else ()):
        ref = interior_from_halo(NAMES[w], o.window(w), d.nx, d.ny, d.nz)
        fl = max(floor.get(w, 0.0) * elapsed, 1e-15)
        assert rel(g.field(NAMES[w]), ref, fl) <= 1e-8, f"window {w} {tag}"


def lockstep(cfg, steps, reset_at=None, coupled=False):
    o = OracleSolver(copy.deepcopy(cfg))
    g = RichardsSolver(copy.deepcopy(cfg))
    try:
        if coupled:
            o.attach_coupling(0.001)
            g.attachCoupling(0.001)
            bath = o.bath_halo()
            eta, _ = cases.coupled_surface(bath)
            dep = eta - bath
            dep[dep <= 0.001] = 0.0
            for name, v in (("eta", eta), ("dept", dep), ("avail", dep)):
                o.set_surface(name, v)
                g.setSurface(name, v)
        o.enable_transport_window()
        g.enableTransportWindow()
        t = 0.0
        elapsed = 0.0
        for n in range(steps):
            dtg = o.next_dt()
            assert g.nextDt() == pytest.approx(dtg, rel=1e-9), n
            t += dtg
            elapsed += dtg
            o.step(t, dtg)
            g.step(t, dtg)
            check(g, o, cfg, f"step {n}", elapsed, vent=coupled)
            if n == reset_at:
                o.reset_transport_window()
                g.resetTransportWindow()
                elapsed = 0.0
                check(g, o, cfg, "reset", dtg, vent=coupled)
        return g.field("win_z"), g.field("qz")
    finally:
        g.close()
        o.close()


@pytest.mark.parametrize("name", ["gravity_bottom", "hydrostatic_side", "mixed_box",
                                  "sand_clay_redistribute"])
def test_window_matches_oracle(name):
    lockstep(cases.SCENARIOS[name](), 10, reset_at=5)


def test_window_coupled_vents_match_oracle():
    lockstep(cases.coupled_box("consistent"), 8, coupled=True)


def test_window_off_by_default_and_batch_refuses_it():
    cfg = cases.SCENARIOS["mixed_box"]()
    a = RichardsSolver(copy.deepcopy(cfg))
    b = RichardsSolver(copy.deepcopy(cfg))
    try:
        with pytest.raises(FatalError):
            a.windowVolumeZ()
        a.enableTransportWindow()
        with pytest.raises(FatalError):
            RichardsBatch([a, b])
    finally:
        a.close()
        b.close()
