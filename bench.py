"""Throughput of the B200 groundwater step (cell-steps/s).

Workload: the terrain-following heterogeneous slab of
``frehg_b200.workloads.hillslope`` (512x512x128 by default, 33.5M cells,
seeded synthetic inputs), one groundwater step (``RichardsSolver::step``:
predictor assembly, Jacobi-PCG head solve, corrector, post-allocation,
clamp, audit, adaptive controller) per timed step, dt driven by the
step's own controller from dt0 = 60 s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
    python bench.py --impl reference ...   # the reference's CPU step, full slab

At N = 1 the line also carries, each measured outside the timed region:
``latency`` (p50 / p99 of the per-step solve and step device times),
``mixed_error`` (the mixed form against the tight FP64 form over a 10-step
trajectory: head, flux, storage, audit, iteration counts, cells whose
theta took the other post-allocation branch; beside it the FP64 form at its
configured rtol against the same tight solve), ``serve`` (a
short Poisson stream through the serving loop: p50 / p99 request latency,
cell-steps/s), ``ensemble`` (a 64-member batch, both forms, against stepping
the members one by one) and ``cpu_baseline`` (the reference's step on
crops, both preconditioner lanes, with CG iteration counts).

With N > 1 the script runs under torchrun, one rank per GPU; every rank
steps its own independent domain (an ensemble member with its own seed), so
the work per GPU is fixed (weak scaling) and there is no data-path
collective; rank 0 prints the line with the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic bytes per active cell (interior cells, each array read or
# written once per pass).
ALG_BYTES_PER_CG_ITER = 128   # FP64 Jacobi-PCG iteration: 16 words
ALG_BYTES_MIXED_INNER = 64    # FP32 inner iteration: stencil pass 10 words (z, p_old,
                              # d, diag, gxp, gyp, gzp in; p, w, d out; d += alpha p of
                              # the previous iteration), update + line solve 6 words
                              # (r, w, dinv, l in; r, z out)
ALG_BYTES_MIXED_FIRST = 12    # less in each inner solve's first iteration (p = z:
                              # neither p_old nor d)
ALG_BYTES_MIXED_SWEEP = 76    # FP64 outer residual sweep: x, b, 4 coefficients, d, l,
                              # dinv in; x, r, z out
ALG_BYTES_MIXED_OUTER = 8     # per correction: its last update's p, read by the next
                              # sweep, and the d reset
ALG_BYTES_MIXED_INIT = 12     # b read for ||b||, d = 0 at entry (the assembly writes
                              # the starting iterate x = h^n)
ALG_BYTES_FIXED = 536         # FP64 step outside the solve
METRIC = "cell-steps/s at 512x512x128"
# DRAM bytes (read + write) per algorithmic byte of k_cg_mixed, from the ncu
# capture summarised in profiles/ (256x256x128 slab, one steady-state launch);
# scaled to the timed launches by their algorithmic bytes.
MIXED_TRAFFIC_PER_ALG_BYTE = 1.023
# Bytes frehg_gw_step reads back per step: the device step record (nine FP64
# audit and controller terms, the solver's exit state, the coupled-top books).
STEP_RECORD_BYTES = 192


def mixed_alg_bytes(cells, inner, outer, launches):
    """Algorithmic bytes of `launches` k_cg_mixed launches that ran `inner`
    inner iterations and `outer` outer corrections in total."""
    sweeps = outer + launches
    return cells * (ALG_BYTES_MIXED_INNER * inner - ALG_BYTES_MIXED_FIRST * outer +
                    ALG_BYTES_MIXED_SWEEP * sweeps + ALG_BYTES_MIXED_OUTER * outer +
                    ALG_BYTES_MIXED_INIT * launches)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                   help="form of the headline value; the other form is timed too")
    p.add_argument("--size", default="512,512,128")
    p.add_argument("--e2e-steps", type=int, default=-1,
                   help="steps of the e2e leg (-1: the timed steps themselves, replayed)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--workload", default="slab", choices=["slab", "ensemble", "serve"],
                   help="slab: the 512x512x128 headline; ensemble: many uneven domains "
                        "stepped as one batch; serve: a Poisson stream of mixed-size "
                        "requests through the serving loop (each prints its own line)")
    p.add_argument("--rates", default="10,100,1000", help="serve: arrival rates, req/s")
    p.add_argument("--requests", type=int, default=64, help="serve: requests per rate")
    p.add_argument("--members", type=int, default=256)
    p.add_argument("--seq-steps", type=int, default=3,
                   help="ensemble: steps of the member-by-member comparison loop")
    p.add_argument("--ref-steps", type=int, default=2,
                   help="reference arm: at most this many timed full-size steps (each takes "
                        "tens of seconds on the host), after one warm-up step")
    p.add_argument("--error-steps", type=int, default=10,
                   help="slab: steps of the mixed-vs-FP64 trajectory behind mixed_error "
                        "(0: skip)")
    p.add_argument("--summary-members", type=int, default=64,
                   help="slab: members of the ensemble summary (0: skip)")
    p.add_argument("--summary-requests", type=int, default=16,
                   help="slab: requests of the served-stream summary (0: skip)")
    p.add_argument("--summary-rate", type=float, default=100.0,
                   help="slab: arrival rate of the served-stream summary, req/s")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.first = threading.Event()
        self.start_n = 0

    def __enter__(self):
        # nvidia-smi's start-up (its NVML initialisation) runs before the
        # region: the region starts once the first sample has arrived, and the
        # summary keeps the samples taken inside it (the pre-region one only
        # when the region was shorter than the sampling period).
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.first.wait(timeout=5.0)
            self.start_n = len(self.lines)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())
            self.first.set()

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        inside = self.lines[self.start_n:]
        for ln in (inside if inside else self.lines):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def slab_config(size: str) -> dict:
    """The workload both arms name in their line's ``config``."""
    nx, ny, nz = (int(v) for v in size.split(","))
    return {"workload": f"terrain-following heterogeneous slab {nx}x{ny}x{nz} "
                        "(hillslope, seeded), dt0 60 s adaptive",
            "active_cells_per_gpu": nx * ny * nz,
            "l2": "inputs larger than L2 (13 GB working set)"}


def ref_lane(size: str, pc: str, threads: int, warmup: int, steps: int):
    """The reference's own CPU step (its src/gw compiled on host shims,
    OpenMP shim backend) on the slab of ``size``: ``warmup`` untimed steps
    (the first, dt0 = 60 s, is the costly one), then ``steps`` timed.  CG
    iterations are reported for the timed steps and for all of them."""
    from frehg_b200 import workloads
    from oracle import ref as refmod
    nx, ny, nz = (int(v) for v in size.split(","))
    cfg = workloads.hillslope(nx, ny, nz)
    os.environ["OMP_NUM_THREADS"] = str(threads)
    t_setup = time.perf_counter()
    r = refmod.RefSolver(cfg, pc=pc, omp=True)
    setup_s = time.perf_counter() - t_setup
    its_all = []
    for _ in range(warmup):
        r.advance()
        its_all.append(r.last_solve()[0])
    its = []
    t0 = time.perf_counter()
    for _ in range(steps):
        r.advance()
        its.append(r.last_solve()[0])
    dt = time.perf_counter() - t0
    _, ktop = r.gid()
    active = int(sum(nz - k for k in ktop.ravel()))
    r.close()
    its_all += its
    return {"value": active * steps / dt, "unit": "cell-steps/s", "size": size, "pc": pc,
            "steps": steps, "warmup": warmup, "s_per_step": dt / steps, "setup_s": setup_s,
            "cg_iterations_mean": sum(its) / len(its), "cg_iterations_max": max(its),
            "cg_iterations_all_steps": its_all}


PC_NAMES = {"icc": "bjacobi-ICC(0) (the reference's default)",
            "jacobi": "Jacobi (-gw_pc_type jacobi, the GPU FP64 form's preconditioner)"}


def cpu_baseline(threads: int):
    """The reference's CPU step on bounded crops of the slab (about 30 s of
    host work): both preconditioner lanes on a 64x64x128 crop and the default
    lane on a 128x128x128 crop, one warm-up and three timed steps each.
    ``value`` is the default lane on the larger crop; the sweep shows how the
    per-cell throughput and the CG counts move with the lateral size (the
    reference arm, ``--impl reference``, times the full slab)."""
    from oracle import ref as refmod
    if not refmod.available(omp=True):
        return None
    lanes = {}
    for size, pc in (("64,64,128", "icc"), ("64,64,128", "jacobi"), ("128,128,128", "icc")):
        lanes[f"{pc}_{size.replace(',', 'x')}"] = ref_lane(size, pc, threads, 1, 3)
    best = lanes["icc_128x128x128"]
    return {"value": best["value"], "unit": "cell-steps/s", "cores": threads,
            "kind": "reference",
            "sample": "128x128x128 crop of the slab, 3 steps after the dt0 = 60 s step, "
                      "reference src/gw on host shims (OpenMP), bjacobi-ICC(0) CG; "
                      "lanes: both preconditioners on a 64x64x128 crop too",
            "lanes": lanes}


def run_reference(args, rank):
    """``--impl reference``: the reference's own step on the host cores, on
    the full slab this arm's line names (setup untimed; one warm-up step, the
    dt0 = 60 s one; then at most ``--ref-steps`` timed steps, since one
    full-size step takes tens of seconds), bjacobi-ICC(0), all host threads."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    from oracle import ref as refmod
    if not refmod.available(omp=True):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref (reference sources on host shims) not built"}))
        return
    steps = max(1, min(args.steps, args.ref_steps))
    res = ref_lane(args.size, "icc", threads, 1, steps)
    sample = (f"the full {args.size.replace(',', 'x')} slab: {steps} timed steps after 1 "
              "warm-up (the dt0 = 60 s step), reference src/gw on host shims (OpenMP), "
              f"{PC_NAMES['icc']} CG")
    line = {
        "metric": METRIC, "value": res["value"], "unit": "cell-steps/s", "n_gpus": args.gpus,
        "steps": steps, "warmup": 1, "steps_requested": args.steps,
        "warmup_requested": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": slab_config(args.size),
        "cpu_baseline": {"kind": "reference", "cores": threads, "sample": sample,
                         "value": res["value"], "unit": "cell-steps/s"},
        "e2e": {"value": res["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "lane": res,
    }
    print(json.dumps(line))


def reduce_over_ranks(dist, ms: float, active: int, device) -> tuple:
    """The job's time (the slowest rank's) and the cells all ranks stepped:
    every rank calls it once after its timed region, in the same order."""
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    a = torch.tensor([float(active)], device=device, dtype=torch.float64)
    dist.all_reduce(a)
    return float(t.item()), float(a.item())


def latency_summary(solve_ms, step_ms) -> dict:
    """p50 / p99 of the per-step device times (CUDA events around each phase
    of every timed step): the predictor solve alone and the whole step."""
    a, b = np.asarray(solve_ms), np.asarray(step_ms)
    return {"solve_p50_ms": float(np.percentile(a, 50)), "solve_p99_ms": float(np.percentile(a, 99)),
            "step_p50_ms": float(np.percentile(b, 50)), "step_p99_ms": float(np.percentile(b, 99)),
            "samples": int(a.size)}


def mixed_error(size: str, steps: int, stream) -> dict:
    """The mixed form against the FP64 form solved tightly (CG rtol 1e-13),
    both on this GPU from the slab's initial state, on the FP64 form's dt
    sequence, never re-synced (``frehg_b200.accuracy``).  Beside it, the
    same comparison for the FP64 form at its configured rtol (the
    reference's own solve, the one the reference ships): the spread the
    reference's tolerance itself allows on this trajectory."""
    import copy

    from frehg_b200 import accuracy, workloads
    from frehg_b200.gw import RichardsSolver

    nx, ny, nz = (int(v) for v in size.split(","))
    cfg = workloads.hillslope(nx, ny, nz)
    own = copy.deepcopy(cfg)
    own.solver.precision = "fp64"
    forms = {"mixed": RichardsSolver(accuracy.mixed(cfg), stream=stream.cuda_stream),
             "fp64": RichardsSolver(own, stream=stream.cuda_stream)}
    ref = RichardsSolver(accuracy.tight_fp64(cfg), stream=stream.cuda_stream)
    try:
        res = accuracy.trajectories(forms, ref, steps, cfg.domain.dx, cfg.domain.dy)
    finally:
        for m in forms.values():
            m.close()
        ref.close()
    s = res["mixed"]
    per = s.pop("per_step")
    s["head_per_step"] = [p["head"] for p in per]
    s["theta_cells_per_step"] = [p["theta_cells"] for p in per]
    env = res["fp64"]
    env.pop("per_step")
    s["fp64_rtol_envelope"] = {
        "rtol": cfg.solver.rtol,
        **{k: env[k] for k in ("head", "flux", "storage", "storage_unflipped", "theta_cells",
                               "audit", "inner_iterations_per_step")}}
    s["reference"] = "FP64 form, Jacobi CG to rtol 1e-13, same dt sequence, no re-sync"
    s["scales"] = {"head": "max(max|h|, 1 m)", "flux": "K A of the face direction",
                   "storage": "owned volume", "audit": "owned volume",
                   "theta_cells": "cells with |theta - theta_ref| > 1e-6"}
    return s


def timed_form(args, precision, rank, local, dist, stream, e2e_steps):
    """Warm-up, then K timed steps of one solver form; optional e2e leg."""
    import torch

    from frehg_b200 import workloads
    from frehg_b200.config import rasterize
    from frehg_b200.gw import RichardsSolver

    nx, ny, nz = (int(v) for v in args.size.split(","))
    cfg = workloads.hillslope(nx, ny, nz, seed=20261203 + rank, precision=precision)
    gw = RichardsSolver(cfg, stream=stream.cuda_stream)
    active = gw.activeCells()
    for _ in range(args.warmup):
        gw.advance()
    # The e2e leg replays the timed steps from this state (the step gets
    # cheaper as the run proceeds, so both legs must time the same steps).
    ck = gw.checkpoint() if e2e_steps else None
    gw.setProfiling(True)
    launches0 = gw.kernelLaunches()
    iters, outer, solve_ms = 0, 0, 0.0
    solve_list, step_list = [], []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            gw.advance()
            iters += gw.lastSolve()[0]
            outer += gw._info["outer_iterations"]
            ph = gw.phaseTimes()
            solve_ms += ph["solve"]
            solve_list.append(ph["solve"])
            step_list.append(sum(ph.values()))
        end.record(stream)
        torch.cuda.synchronize()
    launches = gw.kernelLaunches() - launches0
    ms = start.elapsed_time(end)
    total_cells = float(active)
    if dist:
        ms, total_cells = reduce_over_ranks(dist, ms, active, "cuda")
    out = dict(value=total_cells * args.steps / (ms / 1e3), ms=ms, iters=iters, outer=outer,
               solve_ms=solve_ms, launches=launches, clocks=clocks.summary(), active=active,
               e2e=None, latency=latency_summary(solve_list, step_list))
    if e2e_steps:
        e2e_steps = args.steps if e2e_steps < 0 else e2e_steps
        gw.restore(ck)
        # End to end through the public API, as a driver calls it each step:
        # that step's boundary values uploaded from host memory (the handle's
        # page-locked staging), the step, and its audit record read back.  The
        # fields stay on the device, as the reference keeps them in its views.
        ras = rasterize(cfg)
        vals = (ras.top_value, ras.bot_value, ras.xm_value, ras.xp_value, ras.ym_value,
                ras.yp_value)
        # what the library uploads: the top and bottom slots ((nx+2)(ny+2)
        # each) and the four sides' edge entries
        h2d = (2 * (nx + 2) * (ny + 2) + 2 * ny + 2 * nx) * 8
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            gw.setBoundaryValues(*vals)
            gw.advance()
        e2e_s = time.perf_counter() - t0
        out["e2e"] = {"value": total_cells * e2e_steps / e2e_s, "unit": "cell-steps/s",
                      "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": STEP_RECORD_BYTES,
                      "steps": e2e_steps}
    gw.close()
    return out


def ensemble_forms(members, steps, warmup, seq_steps, rank):
    """Both forms of an ensemble of ``members`` seeded domains: autotune,
    ``warmup`` batch steps, ``steps`` timed batch steps, then ``seq_steps``
    member-by-member steps for comparison."""
    import torch

    from frehg_b200 import workloads
    from frehg_b200.batch import RichardsBatch
    from frehg_b200.gw import RichardsSolver

    forms = {}
    for prec in ("mixed", "fp64"):
        cfgs = workloads.ensemble(members, seed=20261204 + rank, precision=prec)
        solvers = [RichardsSolver(c) for c in cfgs]
        cells = float(sum(s.activeCells() for s in solvers))
        batch = RichardsBatch(solvers)
        tuned, tune_ms = batch.autotune(trials=1)
        for _ in range(warmup):
            batch.step()
        st0 = batch.stats()
        torch.cuda.synchronize()
        with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
            t0 = time.perf_counter()
            iters = 0
            for _ in range(steps):
                infos = batch.step()
                iters += sum(i["cg_iterations"] for i in infos)
            sec = time.perf_counter() - t0
        st = batch.stats()
        batch.close()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(seq_steps):
            for s in solvers:
                s.advance()
        seq_sec = time.perf_counter() - t1
        for s in solvers:
            s.close()
        forms[prec] = {
            "value": cells * steps / sec, "ms_per_step": 1e3 * sec / steps,
            "members": len(cfgs), "active_cells": cells,
            "solve_iterations_per_member_step": iters / (steps * len(cfgs)),
            "kernels_per_step": st["kernels_per_step"],
            "kernel_launches": st["kernel_launches"] - st0["kernel_launches"],
            "solve_launches_per_step": st["solve_launches"], "solve_blocks": st["solve_blocks"],
            "graph_replay": bool(st["uses_graph"]), "autotuned": tuned,
            "autotune_best_step_ms": tune_ms, "clocks": clocks.summary(),
            "member_by_member": {"value": cells * seq_steps / seq_sec,
                                 "ms_per_step": 1e3 * seq_sec / seq_steps,
                                 "steps": seq_steps},
            "batch_over_member_by_member": (cells * steps / sec) /
                                           (cells * seq_steps / seq_sec),
        }
    return forms


def run_ensemble(args, rank, world):
    """Many uneven domains stepped as one batch (frehg_gw_batch_*), each form.

    The members (``workloads.ensemble``: nx, ny ~ U{16..128}, nz ~ U{32..200},
    per-member soil, seeded) are stepped with their own adaptive dt; the batch
    is autotuned first (trial steps from a snapshot, state restored), then
    ``--warmup`` steps, then ``--steps`` timed steps, each ending with the
    batch's host synchronisation, so wall time is device time plus the host's
    step records.  For comparison the same members are then stepped one after
    another through frehg_gw_step for ``--seq-steps`` steps.  Under torchrun
    every rank steps its own ensemble (seed + rank); no collective.
    """
    forms = ensemble_forms(args.members, args.steps, args.warmup, args.seq_steps, rank)
    if rank != 0:
        return
    line = {
        "metric": "cell-steps/s, ensemble of uneven domains stepped as one batch",
        "value": forms["mixed"]["value"], "unit": "cell-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": forms["mixed"]["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32-inner/f64", "data": "synthetic",
        "config": {"workload": f"{args.members} independent boxes, nx,ny U{{16..128}}, "
                               "nz U{32..200}, per-member van Genuchten + lnKs ~ N(ln 1e-5, 1), "
                               "head0 U[-3,-0.2], ponded head or 1e-6 m/s flux top, "
                               "own adaptive dt each",
                   "parallelism": f"replicas x{world}"},
        "forms": forms,
        "mixed_over_fp64": forms["mixed"]["value"] / forms["fp64"]["value"],
    }
    print(json.dumps(line))


def serve_requests(n, seed):
    """``n`` requests: cells log-uniform in [1e4, 1e7], nz ~ U{32..200},
    nx = ny from the cell count, soil and top condition drawn as for the
    ensemble members, steps ~ U{20..200}; mixed precision."""
    from frehg_b200 import workloads

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        cells = float(np.exp(rng.uniform(np.log(1e4), np.log(1e7))))
        nz = int(rng.integers(32, 201))
        side = max(2, int(round(np.sqrt(cells / nz))))
        cfg = workloads.ensemble_member(rng, "mixed", (side, side), (nz, nz))
        out.append((cfg, int(rng.integers(20, 201))))
    return out


def serve_summary(n_requests: int, rate: float, rank: int) -> dict:
    """A short served stream (``n_requests`` of :func:`serve_requests`,
    Poisson arrivals at ``rate`` req/s): p50 / p99 request latency and
    cell-steps/s, for the headline line."""
    from frehg_b200.serve import PreparedRequest, RichardsServer, run_stream

    reqs = [PreparedRequest(c, n) for c, n in serve_requests(n_requests, 20261205 + rank)]
    rng = np.random.default_rng(7 + rank)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs)))
    with RichardsServer() as srv:
        res = run_stream(srv, reqs, arrivals)
    res["rate_req_per_s"] = rate
    res["requested_cell_steps"] = int(sum(r.nx * r.ny * r.nz * r.steps for r in reqs))
    return res


def run_serve(args, rank, world):
    """A Poisson stream of mixed-size requests through frehg_gw_server_*.

    For each arrival rate, ``--requests`` requests (see serve_requests) are
    prepared on the host first, then submitted at seeded exponential
    inter-arrival times while the server ticks (admit by free device memory
    and slots, one batch step of everything admitted, retire); latency is
    submission to completion.  Under torchrun every rank serves its own
    stream; no collective.
    """
    from frehg_b200.serve import PreparedRequest, RichardsServer, run_stream

    rates = [float(r) for r in args.rates.split(",")]
    reqs = [PreparedRequest(c, n) for c, n in serve_requests(args.requests, 20261205 + rank)]
    work = sum(r.nx * r.ny * r.nz * r.steps for r in reqs)
    per_rate = {}
    for rate in rates:
        rng = np.random.default_rng(7 + rank)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs)))
        with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
            with RichardsServer() as srv:
                res = run_stream(srv, reqs, arrivals)
        res["clocks"] = clocks.summary()
        res["arrival_span_s"] = float(arrivals[-1])
        per_rate[str(int(rate) if rate.is_integer() else rate)] = res
    if rank != 0:
        return
    best = max(per_rate.values(), key=lambda r: r["cell_steps_per_s"])
    line = {
        "metric": "served stream: cell-steps/s with p50/p99 request latency",
        "value": best["cell_steps_per_s"], "unit": "cell-steps/s", "n_gpus": world,
        "steps": None, "warmup": 0, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32-inner/f64", "data": "synthetic",
        "config": {"workload": f"{args.requests} requests per rate, cells log-uniform 1e4-1e7, "
                               "nz U{32..200}, 20-200 adaptive steps each, mixed precision, "
                               "Poisson arrivals",
                   "rates_req_per_s": rates, "requested_cell_steps": int(work),
                   "parallelism": f"replicas x{world}"},
        "per_rate": per_rate,
    }
    print(json.dumps(line))


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch

    torch.cuda.set_device(local)
    if args.workload == "ensemble":
        run_ensemble(args, rank, world)
        return
    if args.workload == "serve":
        run_serve(args, rank, world)
        return
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    stream = torch.cuda.Stream()
    other = "fp64" if args.precision == "mixed" else "mixed"
    res_other = timed_form(args, other, rank, local, dist, stream, 0)
    # The mixed form's algorithm with FP64 inner iterations: what FP32 buys.
    res_line = timed_form(args, "fp64_line", rank, local, dist, stream, 0)
    res = timed_form(args, args.precision, rank, local, dist, stream, args.e2e_steps)
    fp64 = res if args.precision == "fp64" else res_other
    mixed = res if args.precision == "mixed" else res_other

    peak, peak_kind = peaks()
    # Roofline of the dominant kernel of each form: its predictor solve, one
    # launch per step, timed by the handle's CUDA events around that launch.
    fp64_ach = (ALG_BYTES_PER_CG_ITER * fp64["active"] * fp64["iters"] /
                (fp64["solve_ms"] / 1e3) / 1e9) if fp64["solve_ms"] else 0.0
    mixed_ach = (mixed_alg_bytes(mixed["active"], mixed["iters"], mixed["outer"], args.steps) /
                 (mixed["solve_ms"] / 1e3) / 1e9) if mixed["solve_ms"] else 0.0
    roof_fp64 = {"bound": "hbm", "kernel": "k_cg64v (FP64 Jacobi-PCG, one launch per step)",
                 "achieved": fp64_ach, "peak": peak, "unit": "GB/s", "frac": fp64_ach / peak,
                 "peak_source": peak_kind, "alg_bytes_per_cell_iter": ALG_BYTES_PER_CG_ITER,
                 "cg_iterations_per_step": fp64["iters"] / args.steps,
                 "solve_share_of_step": fp64["solve_ms"] / fp64["ms"] if fp64["ms"] else None}
    mixed_traffic = None
    if MIXED_TRAFFIC_PER_ALG_BYTE is not None:
        mixed_traffic = MIXED_TRAFFIC_PER_ALG_BYTE * mixed_alg_bytes(
            mixed["active"], mixed["iters"], mixed["outer"], args.steps) / args.steps
    roof_mixed = {"bound": "hbm",
                  "kernel": "k_cg_mixed (FP32 line-PCG inside FP64 defect correction, one "
                            "cooperative launch per step)",
                  "achieved": mixed_ach, "peak": peak, "unit": "GB/s", "frac": mixed_ach / peak,
                  "peak_source": peak_kind, "traffic": mixed_traffic,
                  "alg_bytes_per_cell": {"inner_iteration": ALG_BYTES_MIXED_INNER,
                                         "outer_sweep": ALG_BYTES_MIXED_SWEEP},
                  "inner_iterations_per_step": mixed["iters"] / args.steps,
                  "outer_sweeps_per_step": mixed["outer"] / args.steps,
                  "solve_share_of_step": mixed["solve_ms"] / mixed["ms"] if mixed["ms"] else None}
    roof = roof_mixed if args.precision == "mixed" else dict(roof_fp64, traffic=None)
    forms = {
        "fp64": {"value": fp64["value"], "ms_per_step": fp64["ms"] / args.steps,
                 "cg_iterations_per_step": fp64["iters"] / args.steps,
                 "solve_ms_per_step": fp64["solve_ms"] / args.steps, "roofline": roof_fp64,
                 "latency": fp64["latency"]},
        "mixed": {"value": mixed["value"], "ms_per_step": mixed["ms"] / args.steps,
                  "inner_iterations_per_step": mixed["iters"] / args.steps,
                  "outer_sweeps_per_step": mixed["outer"] / args.steps,
                  "solve_ms_per_step": mixed["solve_ms"] / args.steps, "roofline": roof_mixed,
                  "latency": mixed["latency"]},
        "fp64_line": {"value": res_line["value"], "ms_per_step": res_line["ms"] / args.steps,
                      "inner_iterations_per_step": res_line["iters"] / args.steps,
                      "outer_sweeps_per_step": res_line["outer"] / args.steps,
                      "solve_ms_per_step": res_line["solve_ms"] / args.steps,
                      "solve_alg_bytes_per_cell_inner": 128,
                      "latency": res_line["latency"]},
        "mixed_over_fp64": mixed["value"] / fp64["value"] if fp64["value"] else None,
        # the split of mixed / FP64: precision alone (same algorithm, FP64
        # inner iterations) and the algorithm (line preconditioner + warm
        # start against point Jacobi from x = 0), for the step and the solve
        "mixed_over_fp64_line": mixed["value"] / res_line["value"] if res_line["value"] else None,
        "fp64_line_over_fp64": res_line["value"] / fp64["value"] if fp64["value"] else None,
        "solve_fp64_line_over_mixed": (res_line["solve_ms"] / mixed["solve_ms"]
                                       if mixed["solve_ms"] else None),
        "solve_fp64_over_fp64_line": (fp64["solve_ms"] / res_line["solve_ms"]
                                      if res_line["solve_ms"] else None),
    }
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    extras = {}
    if world == 1:
        # Driver-visible summaries of the rest of the metric (N = 1 only):
        # the mixed form's error against the tight FP64 form over a
        # trajectory, a short served stream (p50 / p99 request latency) and a
        # smaller ensemble batch, each outside the timed region.
        if args.error_steps > 0:
            extras["mixed_error"] = mixed_error(args.size, args.error_steps, stream)
        if args.summary_requests > 0:
            extras["serve"] = serve_summary(args.summary_requests, args.summary_rate, rank)
        if args.summary_members > 0:
            extras["ensemble"] = ensemble_forms(args.summary_members, 5, 3, 2, rank)
            extras["ensemble"]["config"] = (f"{args.summary_members} independent boxes of "
                                            "workloads.ensemble (seeded), 3 warm-up + 5 timed "
                                            "batch steps, 2 member-by-member steps")
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        cpu = cpu_baseline(os.cpu_count() or 1)
    cfg_line = slab_config(args.size)
    cfg_line["active_cells_per_gpu"] = res["active"]
    line = {
        "metric": METRIC, "value": res["value"], "unit": "cell-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32-inner/f64",
        "data": "synthetic",
        "config": cfg_line, "form": args.precision, "parallelism": f"replicas x{world}",
        "roofline": roof, "forms": forms, "cpu_baseline": cpu, "e2e": res["e2e"],
        "gpu_launches": res["launches"], "clocks": res["clocks"],
        "latency": res["latency"],
    }
    line.update(extras)
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
