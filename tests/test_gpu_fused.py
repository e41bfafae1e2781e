"""The fused phase kernels against the separate passes they replace.

A groundwater-only domain with nz <= 256 runs its predictor as one fused
pass by default (closures, faces, rows and, in the mixed form, the column
factors); ``setFused(False)`` runs the separate passes.  Both evaluate the
same closure, face-rule and row functions on the same inputs, so the two
runs agree to rounding at every step; here they are stepped in lockstep and
compared field by field at 1e-13 of each field's scale, with identical CG
iteration counts (a difference in the last bits may change a count by one,
hence +-1).
"""
import numpy as np
import pytest

import cases
from frehg_b200 import workloads
from frehg_b200.gw import RichardsSolver

# The fused passes raised a misaligned-address error on the B200 whose cause
# is not yet found; until it is, they are not run on the GPU.
pytestmark = [pytest.mark.gpu,
              pytest.mark.skip(reason="fused passes off the GPU until a misaligned-address "
                                      "error they raised is understood")]

FIELDS = ("h", "wc", "qx", "qy", "qz", "kx", "ky", "kz")


def lockstep(cfg, steps):
    a, b = RichardsSolver(cfg), RichardsSolver(cfg)
    b.setFused(False)
    bitwise = True
    try:
        for n in range(steps):
            dtg = a.nextDt()
            assert b.nextDt() == pytest.approx(dtg, rel=1e-12), f"dt step {n}"
            a.t += dtg
            b.t += dtg
            ia = a.step(a.t, dtg)
            ib = b.step(b.t, dtg)
            assert abs(ia["cg_iterations"] - ib["cg_iterations"]) <= 1, f"its step {n}"
            for name in FIELDS:
                fa, fb = a.field(name), b.field(name)
                scale = max(float(np.max(np.abs(fb))), 1e-300)
                err = float(np.max(np.abs(fa - fb))) / scale
                assert err <= 1e-13, f"{name} step {n}: {err}"
                bitwise &= bool(np.array_equal(fa, fb))
    finally:
        a.close()
        b.close()
    return bitwise


@pytest.mark.parametrize("name", sorted(cases.SCENARIOS))
def test_fused_equals_separate_scenarios(name):
    lockstep(cases.SCENARIOS[name](), 5)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_equals_separate_slab_crop(precision):
    # nz = 128 (four cells a lane), a partial last strip (nx = 40 is not a
    # multiple of the six interior columns of a block) and a partial last
    # row segment (ny = 37).
    cfg = workloads.hillslope(40, 37, 128, precision=precision)
    lockstep(cfg, 4)


@pytest.mark.parametrize("nz", [20, 50, 200])
def test_fused_equals_separate_depths(nz):
    # one, two and eight cells a lane
    for precision in ("fp64", "mixed"):
        lockstep(workloads.column_32x32x50(nx=9, ny=7, nz=nz, precision=precision), 3)
