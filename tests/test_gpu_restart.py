"""Checkpoint / restart of the groundwater state (frehg_gw_restore).

The reference gates restart determinism: run -> checkpoint -> restart equals
the uninterrupted run (io/Checkpoint.hpp; driver/Simulation.cpp:707-792).
Every other device array is rebuilt within a step, so here the restarted
run must match the uninterrupted one bit for bit, in both solver forms.
"""
import copy

import numpy as np
import pytest

from frehg_b200 import workloads
from frehg_b200.gw import RichardsSolver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_restart_equals_uninterrupted_run(precision, tmp_path):
    cfg = workloads.hillslope(16, 12, 40, n_bumps=3, precision=precision)
    full = RichardsSolver(copy.deepcopy(cfg))
    for _ in range(8):
        full.advance()
    first = RichardsSolver(copy.deepcopy(cfg))
    for _ in range(4):
        first.advance()
    path = str(tmp_path / "gw.npz")
    first.save_checkpoint(path)
    first.close()
    second = RichardsSolver(copy.deepcopy(cfg))   # a fresh run, initial state overwritten
    second.load_checkpoint(path)
    for _ in range(4):
        second.advance()
    assert second.t == full.t
    assert second.nextDt() == full.nextDt()
    for name in ("h", "wc", "vloss", "qz", "qx"):
        np.testing.assert_array_equal(second.field(name), full.field(name), err_msg=name)
    assert second.audit() == full.audit()
    full.close()
    second.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_restart_with_density_coupling(precision, tmp_path):
    # The restart's derived-state refresh recomputes the density ratios from
    # the handed-over scalars before the ghosts (refreshDerivedState,
    # RichardsSolver.cpp:880-890), so hydrostatic edge ghosts and the next
    # step see the running run's ratios.
    import cases

    cfg = cases.SCENARIOS["hydrostatic_side"]()
    cfg.solver.precision = precision
    d = cfg.domain
    kw = dict(saline=True, thermal=True, thermal_expansion=2.0e-4, reallocation_gradient=True)

    def hand(g, n):
        salt, salt_surf, temp, temp_surf = cases.density_scalars(d.nx, d.ny, d.nz, n)
        g.setScalar("salt", salt)
        g.setScalar("salt_surf", salt_surf)
        g.setScalar("temp", temp)
        g.setScalar("temp_surf", temp_surf)

    full = RichardsSolver(copy.deepcopy(cfg))
    full.attachDensity(**kw)
    for n in range(8):
        hand(full, n)
        full.advance()
    first = RichardsSolver(copy.deepcopy(cfg))
    first.attachDensity(**kw)
    for n in range(4):
        hand(first, n)
        first.advance()
    path = str(tmp_path / "gw.npz")
    first.save_checkpoint(path)
    first.close()
    second = RichardsSolver(copy.deepcopy(cfg))
    second.attachDensity(**kw)
    hand(second, 3)  # the scalars of the checkpointed step, as a transport restart restores them
    second.load_checkpoint(path)
    for n in range(4, 8):
        hand(second, n)
        second.advance()
    assert second.nextDt() == full.nextDt()
    for name in ("h", "wc", "vloss", "qz", "qx", "rho_z"):
        np.testing.assert_array_equal(second.field(name), full.field(name), err_msg=name)
    full.close()
    second.close()
