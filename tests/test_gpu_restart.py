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
