"""The mixed-precision form: FP32 inner line-preconditioned CG inside FP64
defect correction (true residual <= 3e-12 ||b||), started from h^n.

Its reference is the FP64 step solved tightly (Jacobi CG, rtol 1e-13): the
default oracle stops its CG at a preconditioned rtol of 1e-8, which leaves
the head itself 1e-7..1e-6 away from the linear system's solution, so a
tighter form is measured against the tight solve.  Two kinds of test:

* one step at a time: the oracle is re-synced to the GPU state before every
  step, so each step's error is measured alone (every scenario);
* trajectories: the two forms step from the same initial state on the same
  dt sequence and are never re-synced, so the error is that of a run -- on a
  64x64x128 crop of the benchmark slab against the tight oracle, and on the
  full 512x512x128 slab against the tight FP64 GPU form.

Bars: head within 1e-8 relative L-inf, the GPU's own mass audit closing to
1e-12 of the total storage.  The trajectories also bound the flux error (on
the gravity scale K A of each direction) and the owned volume's relative
error, and report the iteration counts.
"""
import copy
import json
import os

import numpy as np
import pytest

import cases
from frehg_b200 import accuracy, workloads
from frehg_b200.gw import RichardsSolver
from oracle.gw import OracleSolver

pytestmark = pytest.mark.gpu

H_TOL = 1e-8
AUDIT_TOL = 1e-12
# Trajectory bars for the fluxes (gravity scale) and the owned volume: the
# measured errors sit orders of magnitude below these.
FLUX_TOL = 1e-6
STORAGE_TOL = 1e-10
# Cells whose theta may take the other post-allocation branch: a cell at
# theta_s whose net flux cancels to the solve's residual stays saturated or
# drains to theta(h) by that residual's sign, so any two solves that differ
# by a residual can part there (one cell in ten full-slab steps measured;
# the reference's own FP64 solve at its configured rtol parts in ~38000).
# The volume bar applies to the other cells.
FLIP_MAX = 4
# The mixed form's errors against the tight solve, as a fraction of those of
# the reference's own FP64 solve at its configured rtol.
ENVELOPE_FRAC = 1e-2


def rel_linf(a, b):
    scale = max(float(np.max(np.abs(b))), 1.0)
    return float(np.max(np.abs(a - b)) / scale)


def run(cfg, steps, precision="mixed"):
    cfg = copy.deepcopy(cfg)
    cfg.solver.precision = precision
    tight = copy.deepcopy(cfg)
    tight.solver.precision = "fp64"
    tight.solver.rtol = 1e-13
    tight.solver.atol = 1e-300
    tight.solver.max_iterations = 200000
    gpu = RichardsSolver(cfg)
    cpu = OracleSolver(tight)
    worst = 0.0
    try:
        prev = gpu.ownedVolume()
        t = 0.0
        for n in range(steps):
            cpu.set_state(gpu.head(), gpu.waterContent())
            dtg = gpu.nextDt()
            t += dtg
            info = gpu.step(t, dtg)
            cpu.step(t, dtg)
            # Started from h^n, the solve still takes at least one correction.
            assert info["outer_iterations"] >= 1 and info["status"] == 0
            err = rel_linf(gpu.field("h"), cpu.field("h"))
            worst = max(worst, err)
            assert err <= H_TOL, f"step {n}: head error {err:.3e} vs the tight FP64 solve"
            v = gpu.ownedVolume()
            resid = (v - prev) - (info["boundary_in"] - info["ss_storage"] +
                                  info["realloc_adjust"] - info["vloss"])
            assert abs(resid) <= 1e-12 * max(v, 1.0), f"audit step {n}: {resid}"
            prev = v
    finally:
        gpu.close()
    return worst


@pytest.mark.parametrize("name", ["closed_column_ss", "head_top", "flux_top", "gravity_bottom",
                                  "hydrostatic_side", "side_flux", "sand_clay_redistribute",
                                  "masked_west", "stack_harm", "mixed_box", "terrain_uniform"])
def test_mixed_scenarios(name):
    run(cases.SCENARIOS[name](), 6)


def test_mixed_box_32x32x50():
    run(workloads.column_32x32x50(), 4)


def test_mixed_hillslope_crop():
    run(workloads.hillslope(24, 20, 32), 3)


def test_mixed_hillslope_crop_nz128():
    # The benchmark's column depth: four rows of 32 cells per warp-column solve.
    run(workloads.hillslope(16, 12, 128), 3)


def test_mixed_deep_columns_tiled_solve():
    # Columns deeper than 256 cells take the shared-memory tiled line solve.
    run(workloads.column_32x32x50(nx=4, ny=3, nz=300), 3)


def check_trajectory(s, name):
    out = os.environ.get("FREHG_ACCURACY_OUT")
    if out:
        with open(os.path.join(out, f"mixed_error_{name}.json"), "w") as f:
            json.dump(s, f, indent=1)
    print(name, json.dumps({k: v for k, v in s.items() if k != "per_step"}))
    assert all(p["status"] == 0 for p in s["per_step"])
    assert s["head"] <= H_TOL, s["head"]
    assert s["audit"] <= AUDIT_TOL, s["audit"]
    assert s["flux"] <= FLUX_TOL, s["flux"]
    assert s["theta_cells"] <= FLIP_MAX, s["theta_cells"]
    assert s["storage_unflipped"] <= STORAGE_TOL, s["storage_unflipped"]


def test_mixed_trajectory_slab_crop_vs_oracle():
    # 64x64x128 crop of the benchmark slab, 10 steps, never re-synced,
    # against the oracle solved tightly.
    cfg = workloads.hillslope(64, 64, 128)
    m = RichardsSolver(accuracy.mixed(cfg))
    ref = OracleSolver(accuracy.tight_fp64(cfg))
    try:
        s = accuracy.trajectory(m, ref, 10, cfg.domain.dx, cfg.domain.dy)
    finally:
        m.close()
        ref.close()
    check_trajectory(s, "slab_64x64x128_vs_oracle")


def test_mixed_trajectory_full_slab_vs_fp64():
    # The benchmark's 512x512x128 slab, 10 steps, the mixed form against the
    # FP64 GPU form solved tightly, never re-synced; beside it the FP64 form
    # at its configured rtol against the same tight solve (three solvers on
    # one device, ~45 GB).
    cfg = workloads.hillslope(512, 512, 128)
    own = copy.deepcopy(cfg)
    own.solver.precision = "fp64"
    forms = {"mixed": RichardsSolver(accuracy.mixed(cfg)), "fp64": RichardsSolver(own)}
    ref = RichardsSolver(accuracy.tight_fp64(cfg))
    try:
        res = accuracy.trajectories(forms, ref, 10, cfg.domain.dx, cfg.domain.dy)
    finally:
        for m in forms.values():
            m.close()
        ref.close()
    s, env = res["mixed"], res["fp64"]
    check_trajectory(s, "slab_512x512x128_vs_fp64")
    for k in ("head", "flux", "storage", "theta_cells"):
        assert s[k] <= ENVELOPE_FRAC * env[k], (k, s[k], env[k])


@pytest.mark.parametrize("name", ["head_top", "gravity_bottom", "side_flux", "mixed_box",
                                  "terrain_uniform", "sand_clay_redistribute"])
def test_fp64_line_scenarios(name):
    # The mixed form's algorithm with FP64 inner iterations meets the same
    # bars against the tight FP64 solve.
    run(cases.SCENARIOS[name](), 6, precision="fp64_line")


def test_fp64_line_slab_crop_nz128():
    run(workloads.hillslope(16, 12, 128), 3, precision="fp64_line")
