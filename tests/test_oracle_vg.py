"""The oracle's van Genuchten closures against the reference's hand-computed
golden values (tests/unit/test_vangenuchten.cpp:35-126, 1e-12 relative)."""
import math

import pytest

from oracle.gw import vg

REL = 1.0e-12
WARRICK = (1.43, 1.56, 0.33, 0.0, -0.02)  # alpha, n, theta_s, theta_r, aev
WARRICK_KS = 2.89e-6
SAND = (5.9, 2.68, 0.46, 0.04, -0.02)
SAND_KS = 5.26e-3


def near(actual, expected):
    if expected == 0.0:
        assert actual == 0.0
    else:
        assert actual / expected == pytest.approx(1.0, abs=REL)


def test_theta_warrick():
    near(vg("theta", WARRICK, -10.0), 0.0739753893647920896)
    near(vg("theta", WARRICK, -1.0), 0.229597833180606)
    near(vg("theta", WARRICK, -0.02), 0.329538302833622731)
    assert vg("theta", WARRICK, -0.01) == 0.33  # above aev: saturated
    assert vg("theta", WARRICK, 0.0) == 0.33
    assert vg("theta", WARRICK, 0.5) == 0.33


def test_theta_sand():
    near(vg("theta", SAND, -10.0), 0.0404448494147192347)
    near(vg("theta", SAND, -1.0), 0.0611781812182591983)
    near(vg("theta", SAND, -0.02), 0.459145092411154812)
    assert vg("theta", SAND, -0.01) == 0.46
    assert vg("theta", SAND, 0.0) == 0.46
    assert vg("theta", SAND, 0.5) == 0.46


def test_capacity():
    near(vg("capacity", WARRICK, -10.0), 0.00407832963118645968)
    near(vg("capacity", WARRICK, -1.0), 0.0817714043754333137)
    near(vg("capacity", WARRICK, -0.02), 0.0359170881291010571)
    near(vg("capacity", WARRICK, -0.01), 0.0244480654553699461)  # cutoff at 0, not aev
    assert vg("capacity", WARRICK, 0.0) == 0.0
    assert vg("capacity", WARRICK, 0.5) == 0.0
    near(vg("capacity", SAND, -10.0), 7.47333600479079924e-5)
    near(vg("capacity", SAND, -1.0), 0.0352762354400144718)
    near(vg("capacity", SAND, -0.02), 0.114255158543752424)
    near(vg("capacity", SAND, -0.01), 0.0358164977166531603)
    assert vg("capacity", SAND, 0.0) == 0.0


def test_conductivity():
    near(vg("conductivity", WARRICK, -10.0, WARRICK_KS), 4.2896686667440645e-11)
    near(vg("conductivity", WARRICK, -1.0, WARRICK_KS), 5.420575919043507e-8)
    near(vg("conductivity", WARRICK, -0.02, WARRICK_KS), 2.153644648328222e-6)
    near(vg("conductivity", WARRICK, -0.01, WARRICK_KS), 2.378796558153712e-6)
    assert vg("conductivity", WARRICK, 0.0, WARRICK_KS) == WARRICK_KS
    assert vg("conductivity", WARRICK, 0.5, WARRICK_KS) == WARRICK_KS
    near(vg("conductivity", SAND, -10.0, SAND_KS), 2.1678893902335157e-14)
    near(vg("conductivity", SAND, -1.0, SAND_KS), 3.379411314506458e-8)
    near(vg("conductivity", SAND, -0.02, SAND_KS), 0.004969259950282671)
    near(vg("conductivity", SAND, -0.01, SAND_KS), 0.005169012561134972)
    assert vg("conductivity", SAND, 0.5, SAND_KS) == SAND_KS


def test_head_inversion():
    near(vg("head", WARRICK, 0.033), -42.6502807991778219)
    near(vg("head", SAND, 0.25), -0.220394548940179914)
    assert vg("head", WARRICK, 0.33) == 0.0
    assert vg("head", WARRICK, 0.4) == 0.0
    floored = vg("head", WARRICK, 0.0)
    assert floored == vg("head", WARRICK, -1.0)
    assert floored < -1.0e3 and math.isfinite(floored)
    wc = vg("theta", SAND, -2.5)
    assert vg("head", SAND, wc) / -2.5 == pytest.approx(1.0, abs=1e-10)


def test_conductivity_derivative():
    near(vg("dkdtheta", WARRICK, 0.2, WARRICK_KS), 7.03506545539082082e-7)
    near_sat = vg("dkdtheta", SAND, 0.459999, SAND_KS)
    near(near_sat, 0.635589131661863617)
    assert vg("dkdtheta", SAND, 0.4599999, SAND_KS) == near_sat
