"""Error of the mixed-precision step against an FP64 step over a trajectory.

The mixed form (FP32 inner line-PCG inside FP64 defect correction) and an
FP64 form solved tightly (Jacobi CG to a preconditioned rtol of 1e-13, so
that its own solve error is far below the mixed form's) step from the same
initial state with the same dt sequence -- the FP64 form's controller picks
each dt and both take it -- and are never re-synchronised, so the errors
below are those of a run, not of one step.  Per step it records:

* head: L-inf of the difference over max(max|h|, 1 m);
* flux: for qx, qy, qz the L-inf of the difference over the gravity scale
  K A of that direction (the face conductivity times the face area; a net
  Darcy flux near equilibrium cancels to the solve's residual, so it has
  no scale of its own);
* storage: the owned volume's relative difference, and theta's L-inf;
* theta_cells: how many cells' theta differs by more than 1e-6, and
  storage_unflipped, the relative volume difference over the other cells
  (a cell at theta_s whose net flux cancels to the solve's residual stays
  saturated or drains by the sign of that residual, a difference of order
  theta_s - theta_r in that cell that no tolerance on the solve removes);
* the mixed form's own mass audit, |dV - (in - ss + realloc - vloss)| / V;
* iterations: the mixed form's inner and outer counts, the FP64 form's CG
  count.

Used by the mixed-precision GPU tests and by ``bench.py`` (``mixed_error``).
"""
from __future__ import annotations

import copy

import numpy as np

FLUX_AXES = (("qx", "kx", "ax"), ("qy", "ky", "ay"), ("qz", "kz", None))


def tight_fp64(cfg, rtol: float = 1e-13):
    """The FP64 form of ``cfg`` with its CG solved to ``rtol``."""
    c = copy.deepcopy(cfg)
    c.solver.precision = "fp64"
    c.solver.rtol = rtol
    c.solver.atol = 1e-300
    c.solver.max_iterations = 200000
    return c


def mixed(cfg):
    c = copy.deepcopy(cfg)
    c.solver.precision = "mixed"
    return c


def _rel(a: np.ndarray, b: np.ndarray, scale: float) -> float:
    if not b.size:
        return 0.0
    return float(np.max(np.abs(a - b))) / scale


def step_errors(m, ref, dx: float, dy: float) -> dict:
    """Errors of solver ``m`` against ``ref`` after a step (both expose
    ``field(name)``)."""
    out = {}
    h_ref = ref.field("h")
    out["head"] = _rel(m.field("h"), h_ref, max(float(np.max(np.abs(h_ref))), 1.0))
    wc_ref = ref.field("wc")
    out["theta"] = _rel(m.field("wc"), wc_ref, max(float(np.max(np.abs(wc_ref))), 1e-300))
    flux = 0.0
    for q, k, area in FLUX_AXES:
        a = dx * dy if area is None else ref.field(area)
        scale = max(float(np.max(np.abs(ref.field(k)) * a)), 1e-300)
        e = _rel(m.field(q), ref.field(q), scale)
        out[q] = e
        flux = max(flux, e)
    out["flux"] = flux
    return out


def trajectory(m, ref, steps: int, dx: float, dy: float, t0: float = 0.0) -> dict:
    """Steps ``m`` (mixed) and ``ref`` (FP64) ``steps`` times with ``ref``'s
    dt sequence, never re-syncing.  ``m`` is a :class:`RichardsSolver`
    (its step record carries the iteration counts and the audit terms);
    ``ref`` anything with ``step(t, dtg)``, ``next_dt()``, ``field(name)``,
    ``owned_volume()`` and an ``info`` dict or step record."""
    return trajectories({"m": m}, ref, steps, dx, dy, t0)["m"]


def trajectories(forms: dict, ref, steps: int, dx: float, dy: float, t0: float = 0.0) -> dict:
    """:func:`trajectory` for several solvers at once (name -> solver), all
    on ``ref``'s dt sequence; returns name -> summary.  Besides the errors,
    each step counts the cells whose theta differs from ``ref``'s by more
    than 1e-6 (``theta_cells``): the branches of the post-allocation (a
    cell at theta_s stays saturated or drains to theta(h) by the sign of its
    net inflow) turn a residual-sized difference in a cell whose net flux
    cancels into a difference of order theta_s - theta_r in that one cell,
    and ``storage`` then carries that cell's volume.  ``storage_unflipped``
    is the relative volume difference over the other cells."""
    t = t0
    prev = {n: m.owned_volume() for n, m in forms.items()}
    cell_volume = dx * dy * next(iter(forms.values())).field("dz3d")
    per_step = {n: [] for n in forms}
    for _ in range(steps):
        dtg = ref.next_dt()
        t += dtg
        info_ref = ref.step(t, dtg)
        if info_ref is None:
            info_ref = getattr(ref, "info", {})
        wc_ref = ref.field("wc")
        v_ref = ref.owned_volume()
        for n, m in forms.items():
            info = m.step(t, dtg)
            e = step_errors(m, ref, dx, dy)
            dwc = m.field("wc") - wc_ref
            kept = np.abs(dwc) <= 1e-6
            e["theta_cells"] = int(dwc.size - np.count_nonzero(kept))
            v_m = m.owned_volume()
            e["storage"] = abs(v_m - v_ref) / max(abs(v_ref), 1e-300)
            e["storage_unflipped"] = (abs(float(np.sum(dwc[kept] * cell_volume[kept]))) /
                                      max(abs(v_ref), 1e-300))
            resid = (v_m - prev[n]) - (info["boundary_in"] - info["ss_storage"] +
                                       info["realloc_adjust"] - info["vloss"])
            e["audit"] = abs(resid) / max(v_m, 1.0)
            prev[n] = v_m
            e["inner_iterations"] = int(info["cg_iterations"])
            e["outer_iterations"] = int(info["outer_iterations"])
            e["fp64_iterations"] = int(info_ref["cg_iterations"])
            e["status"] = int(info["status"])
            e["dtg"] = dtg
            per_step[n].append(e)
    return {n: summarize(p) for n, p in per_step.items()}


def summarize(per_step: list) -> dict:
    keys = ("head", "theta", "qx", "qy", "qz", "flux", "storage", "storage_unflipped", "audit",
            "theta_cells")
    s = {k: max(p[k] for p in per_step) for k in keys}
    n = len(per_step)
    s["steps"] = n
    s["inner_iterations_per_step"] = sum(p["inner_iterations"] for p in per_step) / n
    s["outer_iterations_per_step"] = sum(p["outer_iterations"] for p in per_step) / n
    s["fp64_iterations_per_step"] = sum(p["fp64_iterations"] for p in per_step) / n
    s["per_step"] = per_step
    return s
