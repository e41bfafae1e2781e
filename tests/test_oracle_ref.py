"""Pin the C oracle against the reference's own groundwater sources.

``oracle/_ref/libfrehg_ref.so`` is the reference's unmodified src/gw (and the
core/bc/io files it needs) compiled on host shims; the restatement must
reproduce it bit for bit: every field, every audit term, every CG iteration
count and the controller's next dt, step after step.
"""
import numpy as np
import pytest

from cases import SCENARIOS
from frehg_b200 import workloads
from oracle import ref as refmod
from oracle.gw import OracleSolver

pytestmark = pytest.mark.skipif(not refmod.available(), reason="oracle/_ref not built")

FIELDS = ("h", "wc", "qx", "qy", "qz", "kx", "ky", "kz", "wcn")
AUDIT = ("boundary_in", "ss_storage", "realloc_adjust", "realloc_dropped", "vloss")


def run_pair(cfg, steps):
    r = refmod.RefSolver(cfg, pc="jacobi")
    o = OracleSolver(cfg)
    for name in ("dz3d", "bot3d", "ax", "ay", "sinx", "cosx", "siny", "cosy", "h", "wc"):
        np.testing.assert_array_equal(o.field(name), r.field(name), err_msg=name)
    for n in range(steps):
        r.advance()
        o.advance()
        its, res = r.last_solve()
        assert o.info["cg_iterations"] == its, f"step {n}"
        assert o.info["residual_norm"] == res, f"step {n}"
        assert o.next_dt() == r.next_dt(), f"step {n}"
        a = r.audit()
        for k in AUDIT:
            assert o.info[k] == a[k], f"{k} step {n}"
        for name in FIELDS:
            np.testing.assert_array_equal(o.field(name), r.field(name), err_msg=f"{name} step {n}")
        assert o.owned_volume() == r.owned_volume()


@pytest.mark.parametrize("name", sorted(SCENARIOS))
def test_scenario_bitwise(name):
    run_pair(SCENARIOS[name](), 12)


def test_gid_and_masks_match():
    cfg = SCENARIOS["mixed_box"]()
    r = refmod.RefSolver(cfg, pc="jacobi")
    o = OracleSolver(cfg)
    gr, kr = r.gid()
    go, ko = o.gid()
    np.testing.assert_array_equal(go, gr)
    np.testing.assert_array_equal(ko, kr)
    # The product's polygon rasterization equals the reference BoundarySet.
    from frehg_b200.config import rasterize
    ras = rasterize(cfg)
    codes, vals = r.bc_masks(0.0)
    ny, nx = cfg.domain.ny, cfg.domain.nx
    np.testing.assert_array_equal(ras.top_code, codes[0, 1:-1, 1:-1])
    np.testing.assert_array_equal(ras.bot_code, codes[1, 1:-1, 1:-1])
    np.testing.assert_array_equal(ras.xm_code, codes[2, 1:-1, 1])
    np.testing.assert_array_equal(ras.xp_code, codes[3, 1:-1, nx])
    np.testing.assert_array_equal(ras.ym_code, codes[4, 1, 1:-1])
    np.testing.assert_array_equal(ras.yp_code, codes[5, ny, 1:-1])
    np.testing.assert_array_equal(ras.top_value, vals[0, 1:-1, 1:-1])
    np.testing.assert_array_equal(ras.bot_value, vals[1, 1:-1, 1:-1])
    off = r.elevation_offset()
    hyd = ras.xm_code == 4
    np.testing.assert_array_equal(np.where(hyd, ras.xm_value + off, ras.xm_value),
                                  vals[2, 1:-1, 1])


def test_box_32x32x50_bitwise():
    run_pair(workloads.column_32x32x50(), 3)


def test_hillslope_crop_bitwise():
    run_pair(workloads.hillslope(16, 12, 24, per_cell_soil=False), 4)
