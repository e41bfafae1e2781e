"""Pin the oracle's transport window against the reference's own sources.

With the window on (RichardsSolver::enableTransportWindow), every step adds
the face volumes q dtg of all x, y and z face slots into the window, and the
post-allocation walks record each transfer on every face it crosses (the
z window carries those path records; the step's qz keeps the legacy
receiver-face mirror); a coupled column's vents add to the vent window.
The restatement must reproduce the windows bit for bit across steps and a
reset, on scenarios whose walks deposit up, release through a head top, send
down and vent onto a coupled surface.
"""
import numpy as np
import pytest

import cases
from oracle import ref as refmod
from oracle.gw import OracleSolver

pytestmark = pytest.mark.skipif(not refmod.available(), reason="oracle/_ref not built")

WINDOWS = ("x", "y", "z")


def compare(r, o, tag, vent=False):
    for name in WINDOWS + (("vent",) if vent else ()):
        np.testing.assert_array_equal(o.window(name), r.window(name), err_msg=f"{name} {tag}")
    for name in ("h", "wc", "qz"):
        np.testing.assert_array_equal(o.field(name), r.field(name), err_msg=f"{name} {tag}")


@pytest.mark.parametrize("name", ["gravity_bottom", "hydrostatic_side", "sand_clay_drop",
                                  "sand_clay_redistribute", "mixed_box", "ponded_consistent"])
def test_window_bitwise(name):
    cfg = cases.SCENARIOS[name]()
    r = refmod.RefSolver(cfg, pc="jacobi")
    o = OracleSolver(cfg)
    r.enable_transport_window()
    o.enable_transport_window()
    moved = 0.0
    for n in range(10):
        r.advance()
        o.advance()
        compare(r, o, f"step {n}")
        moved = max(moved, float(np.max(np.abs(o.window("z") - 0.0))))
        if n == 5:  # the driver consumes the window and starts the next one
            r.reset_transport_window()
            o.reset_transport_window()
            compare(r, o, "reset")
    assert moved > 0.0


@pytest.mark.parametrize("name", ["gravity_bottom", "hydrostatic_side"])
def test_window_path_records_differ_from_the_legacy_mirror(name):
    # In these columns a walk crosses faces other than its receiver's, so the
    # z window is not the time integral of the step's qz alone.
    cfg = cases.SCENARIOS[name]()
    o = OracleSolver(cfg)
    o.enable_transport_window()
    integral = None
    gap = 0.0
    for n in range(10):
        dtg = o.next_dt()
        o.t += dtg
        o.step(o.t, dtg)
        q = o.field("qz") * dtg
        integral = q if integral is None else integral + q
        gap = max(gap, float(np.max(np.abs(o.window("z")[1:-1, 1:-1, :] - integral))))
    assert gap > 1e-13


def test_window_coupled_vents_bitwise():
    cfg = cases.coupled_box("consistent")
    r = refmod.RefSolver(cfg, pc="jacobi")
    o = OracleSolver(cfg)
    for x in (r, o):
        x.attach_coupling(0.001)
        x.enable_transport_window()
    bath = r.halo_field("bath")
    eta, _ = cases.coupled_surface(bath)
    d = eta - bath
    d[d <= 0.001] = 0.0
    for x in (r, o):
        x.set_surface("eta", eta)
        x.set_surface("dept", d)
        x.set_surface("avail", d)
    for n in range(8):
        r.advance()
        o.advance()
        compare(r, o, f"step {n}", vent=True)
    assert np.max(o.window("vent")) > 0.0
