"""The trajectory comparator (frehg_b200.accuracy) on the CPU: oracle against
oracle, and a planted theta difference in one cell that the comparator has to
count as one branch-parted cell and keep out of storage_unflipped."""
import numpy as np

from frehg_b200 import accuracy, workloads
from oracle.gw import OracleSolver


def _box():
    return workloads.column_32x32x50(nx=4, ny=3, nz=20)


def test_identical_forms_have_zero_error():
    cfg = _box()
    ref, m = OracleSolver(cfg), OracleSolver(cfg)
    try:
        s = accuracy.trajectories({"m": m}, ref, 3, cfg.domain.dx, cfg.domain.dy)["m"]
    finally:
        ref.close()
        m.close()
    for k in ("head", "theta", "flux", "storage", "storage_unflipped"):
        assert s[k] == 0.0, (k, s[k])
    assert s["theta_cells"] == 0
    assert s["steps"] == 3 and len(s["per_step"]) == 3
    assert s["audit"] < 1e-12


def test_planted_cell_is_counted_and_kept_out_of_the_volume_bar():
    # An unsaturated cell deep in the box wetted by 0.2 before the run: its
    # theta stays apart from the reference's, the rest barely moves.
    cfg = _box()
    ref, m = OracleSolver(cfg), OracleSolver(cfg)
    try:
        h, wc = m.field("h"), m.field("wc")
        wc[1, 2, 3] += 0.2
        m.set_state(h, wc)
        s = accuracy.trajectories({"m": m}, ref, 2, cfg.domain.dx, cfg.domain.dy)["m"]
    finally:
        ref.close()
        m.close()
    assert s["theta_cells"] >= 1
    assert np.isfinite(s["storage"]) and s["storage"] > 10 * s["storage_unflipped"]
