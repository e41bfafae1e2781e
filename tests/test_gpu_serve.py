"""The serving loop (frehg_gw_server_*): continuous batching of mixed-size
Richards solves.

A request's result must not depend on what else the server is doing: its
device state, solve decomposition and dt sequence are its own, so a request
run alone and the same request admitted mid-stream among others give the same
head and water content bit for bit.  Against the single-domain step the bar
is the mixed form's parity bar (head within 1e-8 relative).  Admission never
holds more device memory than the budget.
"""
import copy

import numpy as np
import pytest

from frehg_b200 import workloads
from frehg_b200.gw import RichardsSolver
from frehg_b200.serve import DONE, PreparedRequest, RichardsServer

pytestmark = pytest.mark.gpu


def rel_linf(a, b):
    scale = max(float(np.max(np.abs(b))), 1.0)
    return float(np.max(np.abs(a - b)) / scale)


def probe():
    return workloads.column_32x32x50(nx=8, ny=7, nz=40, precision="mixed"), 6


def others():
    return [(workloads.hillslope(10, 8, 64, n_bumps=2, precision="mixed"), 5),
            (workloads.column_32x32x50(nx=6, ny=6, nz=130), 4),
            (workloads.column_32x32x50(nx=5, ny=9, nz=33, precision="mixed"), 7),
            (workloads.hillslope(12, 6, 190, n_bumps=1, precision="mixed"), 3)]


def test_result_same_alone_and_in_the_mix():
    cfg, steps = probe()
    with RichardsServer() as srv:
        rid = srv.submit(cfg, steps)
        srv.run_until_idle()
        st = srv.poll(rid)
        assert st["state"] == DONE and st["steps_done"] == steps
        alone = srv.result(rid)
    with RichardsServer(max_active=3) as srv:
        ids = [srv.submit(c, n) for c, n in others()[:2]]
        srv.tick()
        rid = srv.submit(cfg, steps)          # arrives while others run
        srv.tick()
        ids += [srv.submit(c, n) for c, n in others()[2:]]
        srv.run_until_idle()
        for i in ids + [rid]:
            assert srv.poll(i)["state"] == DONE
        mixed = srv.result(rid)
    for k in ("h", "wc"):
        np.testing.assert_array_equal(mixed[k], alone[k])
    solo = RichardsSolver(copy.deepcopy(cfg))
    for _ in range(steps):
        solo.advance()
    assert rel_linf(alone["h"], solo.field("h")) <= 1e-8
    assert abs(srv_time(cfg, steps) - solo.t) <= 1e-9 * solo.t
    solo.close()


def srv_time(cfg, steps):
    with RichardsServer() as srv:
        rid = srv.submit(cfg, steps)
        srv.run_until_idle()
        return srv.poll(rid)["sim_time"]


def test_admission_keeps_within_the_memory_budget():
    reqs = [PreparedRequest(c, n) for c, n in others()]
    budget = max(r.device_bytes() for r in reqs) + 1024
    assert sum(r.device_bytes() for r in reqs) > budget
    with RichardsServer(hbm_budget_bytes=budget) as srv:
        ids = [srv.submit(r) for r in reqs]
        most = 0
        for _ in range(10000):
            a, q = srv.tick()
            st = srv.stats()
            assert st["device_bytes_used"] <= budget
            most = max(most, a)
            if a == 0 and q == 0:
                break
        # The budget fits the largest request, never all of them at once.
        assert 1 <= most < len(reqs)
        for i, (c, n) in zip(ids, others()):
            p = srv.poll(i)
            assert p["state"] == DONE and p["steps_done"] == n
            assert p["latency_s"] >= p["queue_s"] >= 0.0


def test_device_bytes_estimate_covers_the_allocation():
    import torch
    # A single-soil box (every soil field uniform: one value each) and a
    # per-cell soil slab crop (ksx = ksy = ksz shared, alpha and n per cell).
    cases = [workloads.column_32x32x50(nx=64, ny=48, nz=96, precision=prec)
             for prec in ("fp64", "mixed")]
    cases.append(workloads.hillslope(64, 48, 96, precision="mixed"))
    for cfg in cases:
        prec = cfg.solver.precision
        need = PreparedRequest(cfg, 1).device_bytes()
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        s = RichardsSolver(cfg)
        free1, _ = torch.cuda.mem_get_info()
        used = free0 - free1
        s.close()
        # One arena per handle: the estimate is the allocation, to a page
        # (the handle's stream may take one more).
        assert used <= need + (2 << 20), (prec, used, need)
        assert need <= used + (4 << 20), (prec, used, need)
