"""The reference's groundwater unit-test invariants (tests/unit/test_gw.cpp),
asserted on the CPU oracle: conservation, the audit identity, every boundary
kind, use_full3d, the post-allocation modes, the adaptive controller, masked
columns and the mesh geometry."""
import numpy as np
import pytest

import cases
from oracle.gw import OracleSolver, vg

SAND = (5.9, 2.68, 0.46, 0.04, -0.02)


def audit_residual(prev, v, a, with_realloc=True):
    adj = a["realloc_adjust"] if with_realloc else 0.0
    return (v - prev) - (a["boundary_in"] - a["ss_storage"] + adj - a["vloss"])


def test_closed_column_conserves():  # test_gw.cpp:147-166
    s = OracleSolver(cases.closed_column())
    v0 = prev = s.owned_volume()
    for _ in range(50):
        s.advance()
        v = s.owned_volume()
        assert abs(v - prev) <= 1e-8 * v0
        assert s.info["boundary_in"] == 0.0
        prev = v
    wc = s.field("wc")
    assert wc[0, 0, 19] > 0.2 and wc[0, 0, 0] < 0.2


def test_audit_identity_with_storage():  # :168-186
    s = OracleSolver(cases.closed_column(1e-4))
    prev = s.owned_volume()
    for _ in range(30):
        s.advance()
        v = s.owned_volume()
        assert abs(audit_residual(prev, v, s.info)) <= 1e-12 * max(v, 1.0)
        prev = v


def test_head_top_infiltrates():  # :192-212
    s = OracleSolver(cases.head_top())
    v0 = s.owned_volume()
    inflow = 0.0
    for _ in range(40):
        s.advance()
        inflow += s.info["boundary_in"]
    assert inflow > 0.0 and s.owned_volume() > v0
    assert s.field("wc")[0, 0, 0] > 0.12


def test_flux_top_exact_volume():  # :214-229
    s = OracleSolver(cases.flux_top())
    v0 = s.owned_volume()
    elapsed = sum(s.advance() for _ in range(40))
    expected = 1.0e-6 * elapsed
    assert s.owned_volume() - v0 == pytest.approx(expected, abs=1e-12 * max(expected, 1.0))


def test_gravity_bottom_drains_at_ks():  # :231-264
    s = OracleSolver(cases.gravity_bottom())
    v0 = s.owned_volume()
    dtg = s.advance()
    assert s.info["boundary_in"] == pytest.approx(-1.0e-5 * dtg, abs=1e-18)
    assert abs(audit_residual(v0, s.owned_volume(), s.info)) <= 1e-12
    assert s.owned_volume() < v0


def test_flux_bottom_injects():  # :266-285
    s = OracleSolver(cases.flux_bottom())
    v0 = s.owned_volume()
    elapsed = sum(s.advance() for _ in range(20))
    assert s.owned_volume() - v0 == pytest.approx(2.0e-6 * elapsed, abs=1e-12)


def test_hydrostatic_side_holds():  # :287-321
    s = OracleSolver(cases.hydrostatic_side())
    h0 = s.field("h")
    for _ in range(10):
        s.advance()
    assert np.max(np.abs(s.field("h") - h0)) <= 1e-6


def test_side_flux_positive_inflow():  # :323-345
    s = OracleSolver(cases.side_flux())
    v0 = s.owned_volume()
    elapsed = sum(s.advance() for _ in range(20))
    assert s.owned_volume() - v0 == pytest.approx(4.0e-6 * 0.5 * elapsed, abs=1e-12)


def test_use_full3d_gates_lateral_flow():  # :351-373
    for flag in (False, True):
        s = OracleSolver(cases.full3d(flag))
        s.advance()
        q = s.field("qx")[0, 1, 1] / s.field("ax")[0, 1, 1]
        assert (q != 0.0) if flag else (q == 0.0)


def test_reallocation_surplus_modes():  # :375-434
    dropped = {}
    for redistribute in (False, True):
        s = OracleSolver(cases.sand_over_clay(redistribute))
        v0 = prev = s.owned_volume()
        total = 0.0
        for _ in range(200):
            s.advance()
            v = s.owned_volume()
            assert abs(audit_residual(prev, v, s.info)) <= 1e-12
            total += s.info["realloc_dropped"]
            prev = v
        assert s.owned_volume() > v0
        dropped[redistribute] = total
    assert dropped[False] > 1e-5
    assert dropped[True] <= 1e-9


def test_reallocation_off_is_exactly_conservative():  # :436-472
    s = OracleSolver(cases.sand_over_clay(False, off=True, pc="consistent"))
    v0 = prev = s.owned_volume()
    for _ in range(200):
        s.advance()
        v = s.owned_volume()
        assert s.info["realloc_adjust"] == 0.0 and s.info["realloc_dropped"] == 0.0
        assert abs(audit_residual(prev, v, s.info, with_realloc=False)) <= 1e-12
        prev = v
    assert s.owned_volume() > v0


def test_adaptive_step_grows_and_clamps():  # :506-528
    s = OracleSolver(cases.adaptive_column())
    assert s.next_dt() == 0.1
    s.advance()
    assert s.next_dt() == pytest.approx(0.125, abs=1e-12)
    dtg = 0.0
    for _ in range(30):
        dtg = s.advance()
        assert 0.1 <= s.next_dt() <= 1.0
    assert dtg == 1.0


def test_isolated_cells_restore_head():  # :530-545
    s = OracleSolver(cases.closed_column())
    cfg = cases.base(1, 1, 10, 0.05, 0.5)
    s = OracleSolver(cfg)
    s.advance()
    wc, h = s.field("wc"), s.field("h")
    for k in range(2, 8):
        assert h[0, 0, k] == pytest.approx(vg("head", SAND, wc[0, 0, k]), abs=1e-12)


@pytest.mark.parametrize("pos", [(1, 0), (1, 2), (0, 1), (2, 1)])
def test_masked_column_is_inert(pos):  # :547-615
    s = OracleSolver(cases.masked_column(*pos))
    gid, ktop = s.gid()
    assert ktop[pos] == 4 and s.active_cells() == 32
    wc0, h0 = s.field("wc")[pos], s.field("h")[pos]
    v0 = prev = s.owned_volume()
    for _ in range(30):
        s.advance()
        v = s.owned_volume()
        assert abs(audit_residual(prev, v, s.info)) <= 1e-12
        assert s.info["boundary_in"] == 0.0
        assert abs(v - prev) <= 1e-8 * v0
        prev = v
    np.testing.assert_array_equal(s.field("wc")[pos], wc0)
    np.testing.assert_array_equal(s.field("h")[pos], h0)
    assert s.field("wc")[1, 1, 3] > 0.2 and s.field("wc")[1, 1, 0] < 0.2


def test_regular_mesh_partial_cells():  # :621-645
    s = OracleSolver(cases.regular_partial_cells())
    _, ktop = s.gid()
    assert list(ktop[0]) == [0, 0, 1]
    assert s.elevation_offset() == 0.09
    dz = s.field("dz3d")
    assert dz[0, 0, 0] == pytest.approx(0.1, abs=1e-14)
    assert dz[0, 1, 0] == pytest.approx(0.05, abs=1e-14)
    assert dz[0, 2, 1] == pytest.approx(0.11, abs=1e-14)


def test_terrain_scaled_metrics():  # :647-676
    s = OracleSolver(cases.terrain(False))
    assert s.elevation_offset() == 0.1
    dz = s.field("dz3d")
    assert dz[0, 0, 0] == pytest.approx(0.1, abs=1e-14)
    assert dz[0, 1, 0] == pytest.approx(0.075, abs=1e-14)
    zc0, zc1 = 0.1 - 0.05, 0.0 - 0.5 * 0.075
    hd = abs(zc1 - zc0)
    dist = np.sqrt(hd * hd + 1.0)
    assert s.field("sinx")[0, 1, 0] == pytest.approx(hd / dist, abs=1e-12)
    assert s.field("cosx")[0, 1, 0] == pytest.approx(1.0 / dist, abs=1e-12)
    assert s.field("ax")[0, 1, 0] == pytest.approx(0.5 * (0.1 + 0.075) / dist, abs=1e-12)


def test_terrain_uniform_layers():  # :678-712
    s = OracleSolver(cases.terrain(True))
    np.testing.assert_allclose(s.field("dz3d"), 0.1, atol=1e-14)
    bot = s.field("bot3d")
    assert bot[0, 0, 3] == pytest.approx(0.1 - 0.4, abs=1e-14)
    assert bot[0, 1, 3] == pytest.approx(0.0 - 0.4, abs=1e-14)
    assert s.field("sinx")[0, 1, 0] == pytest.approx(0.1 / np.sqrt(1.01), abs=1e-12)


@pytest.mark.parametrize("harmonic", [False, True])
def test_consistent_pair_books_nothing(harmonic):  # :833-876 (K1)
    s = OracleSolver(cases.heterogeneous_stack(harmonic))
    thr = churn = 0.0
    for _ in range(20):
        dtg = s.advance()
        thr += abs(s.field("qz")[0, 0, 3]) * dtg
        churn += abs(s.info["realloc_adjust"]) + 2.0 * s.info["realloc_dropped"]
    assert thr > 1e-5
    assert churn <= 1e-10 * thr


def test_legacy_pair_churns():  # :878-916
    s = OracleSolver(cases.heterogeneous_stack(False, "legacy"))
    thr = churn = 0.0
    for _ in range(20):
        dtg = s.advance()
        thr += abs(s.field("qz")[0, 0, 3]) * dtg
        churn += abs(s.info["realloc_adjust"]) + 2.0 * s.info["realloc_dropped"]
    assert thr > 1e-5 and churn > 1e-4 * thr


def test_homogeneous_consistent_equals_legacy():  # :918-943 (K3)
    heads = []
    for pc in ("legacy", "consistent"):
        s = OracleSolver(cases.homogeneous_pair(pc))
        for _ in range(30):
            s.advance()
        heads.append(s.field("h")[0, 0])
    np.testing.assert_array_equal(heads[0], heads[1])


def test_ponded_top_consistent_equals_legacy():  # :945-975 (K2)
    th = []
    for pc in ("legacy", "consistent"):
        s = OracleSolver(cases.ponded_top(pc))
        for _ in range(50):
            s.advance()
        th.append(s.field("wc")[0, 0])
    np.testing.assert_array_equal(th[0], th[1])
