"""Batched stepping (frehg_gw_batch_*) against the single-domain step.

Each member of a batch must step exactly as the same domain stepped on its
own: same physics, its own dt, its own solve.  The solve's block count differs
between the two paths (one member of a shared cooperative launch against the
whole device), which changes only the order of the CG reductions, so the
bars are the single-domain parity bars: head within 1e-9 relative L-inf for
the FP64 form and 1e-8 for the mixed form, CG iterations within +/-2, and each
member's own mass audit closing to 1e-12 of its storage.  Within the batch
path the arithmetic is fixed by the member alone: graph replay and direct
launches agree bit for bit, and so does a member alone and in a mix (the
members' solves share one launch per solve kind, their blocks taking block
slots from a queue ranked by the previous step's work, so a member's place in
the queue changes which blocks run it, never its arithmetic).
"""
import copy

import numpy as np
import pytest

import cases
from frehg_b200 import workloads
from frehg_b200.batch import RichardsBatch
from frehg_b200.gw import RichardsSolver

pytestmark = pytest.mark.gpu


def rel_linf(a, b):
    scale = max(float(np.max(np.abs(b))), 1.0)
    return float(np.max(np.abs(a - b)) / scale)


def mix_configs():
    """Members of uneven size, both precisions, odd and even depths,
    column-solve depths 20..190 and the tiled depth 300."""
    out = []
    c = workloads.column_32x32x50(nx=6, ny=5, nz=20)
    out.append(c)
    c = workloads.column_32x32x50(nx=7, ny=4, nz=37, precision="mixed")
    out.append(c)
    out.append(workloads.hillslope(10, 8, 64, n_bumps=2))
    c = workloads.hillslope(9, 7, 128, n_bumps=2, precision="mixed")
    out.append(c)
    c = workloads.column_32x32x50(nx=4, ny=3, nz=300, precision="mixed")
    out.append(c)
    c = cases.SCENARIOS["sand_clay_redistribute"]()
    out.append(c)
    out.append(workloads.column_32x32x50(nx=3, ny=3, nz=190, precision="mixed"))
    return out


def tol(cfg):
    return 1e-8 if cfg.solver.precision == "mixed" else 1e-9


def test_batch_members_match_single_domain_steps():
    cfgs = mix_configs()
    solo = [RichardsSolver(copy.deepcopy(c)) for c in cfgs]
    mem = [RichardsSolver(copy.deepcopy(c)) for c in cfgs]
    batch = RichardsBatch(mem, cells_per_block=2048)
    try:
        prev = [m.ownedVolume() for m in mem]
        for step in range(4):
            infos = batch.step()
            for i, (s, m, cfg) in enumerate(zip(solo, mem, cfgs)):
                s.advance()
                assert abs(m.t - s.t) <= 1e-12 * max(1.0, s.t), (i, m.t, s.t)
                err = rel_linf(m.field("h"), s.field("h"))
                assert err <= tol(cfg), f"member {i} step {step}: head {err:.3e}"
                assert abs(infos[i]["cg_iterations"] - s.lastSolve()[0]) <= 2
                v = m.ownedVolume()
                a = infos[i]
                resid = (v - prev[i]) - (a["boundary_in"] - a["ss_storage"] +
                                         a["realloc_adjust"] - a["vloss"])
                assert abs(resid) <= 1e-12 * max(v, 1.0), (i, step, resid)
                prev[i] = v
        st = batch.stats()
        assert st["members"] == len(cfgs)
        assert st["steps"] == 4
        assert st["kernels_per_step"] > 0
        # Members of every column class share one solve launch per solve kind
        # (FP64 and mixed here), whatever their depths.
        assert st["solve_launches"] == 2, st
    finally:
        batch.close()
        for s in solo + mem:
            s.close()


def run_batch(cfgs, steps, **opts):
    mem = [RichardsSolver(copy.deepcopy(c)) for c in cfgs]
    batch = RichardsBatch(mem, **opts)
    try:
        for _ in range(steps):
            batch.step()
        out = [(m.field("h"), m.field("wc"), m.field("qz")) for m in mem]
        stats = batch.stats()
    finally:
        batch.close()
        for m in mem:
            m.close()
    return out, stats


def test_graph_replay_equals_direct_launches():
    cfgs = mix_configs()[:4]
    a, sa = run_batch(cfgs, 3, cells_per_block=4096, use_graph=True)
    b, sb = run_batch(cfgs, 3, cells_per_block=4096, use_graph=False)
    assert sa["uses_graph"] == 1 and sa["graphs"] >= 1
    assert sb["uses_graph"] == 0
    for x, y in zip(a, b):
        for u, v in zip(x, y):
            np.testing.assert_array_equal(u, v)


def test_batched_phases_equal_member_by_member_launches():
    # One launch per phase for all members gives each member its
    # single-domain block counts, so it must match the per-member launches
    # bit for bit (step records included).
    cfgs = mix_configs()
    a, sa = run_batch(cfgs, 3, cells_per_block=4096)
    b, sb = run_batch(cfgs, 3, cells_per_block=4096, per_member_phases=True)
    assert sa["kernels_per_step"] < sb["kernels_per_step"]
    for x, y in zip(a, b):
        for u, v in zip(x, y):
            np.testing.assert_array_equal(u, v)


def test_member_alone_equals_member_in_mix():
    cfgs = mix_configs()
    alone, _ = run_batch([cfgs[3]], 3, cells_per_block=2048)
    mixed, _ = run_batch(cfgs, 3, cells_per_block=2048)
    for u, v in zip(alone[0], mixed[3]):
        np.testing.assert_array_equal(u, v)


def test_set_members_keeps_every_member_exact():
    # Rebinding the batch mid-run (a member joins, another leaves) changes no
    # member's arithmetic: each ends as it would stepping in a batch alone.
    cfgs = mix_configs()[:3]
    ref, _ = run_batch([cfgs[0]], 4, cells_per_block=4096)
    ref2, _ = run_batch([cfgs[2]], 2, cells_per_block=4096)
    mem = [RichardsSolver(copy.deepcopy(c)) for c in cfgs]
    batch = RichardsBatch(mem[:2], cells_per_block=4096)
    try:
        batch.step()
        batch.step()
        batch.set_members([mem[0], mem[2]])    # member 1 leaves, member 2 joins
        batch.step()
        batch.step()
        for u, v in zip(ref[0], (mem[0].field("h"), mem[0].field("wc"), mem[0].field("qz"))):
            np.testing.assert_array_equal(v, u)
        for u, v in zip(ref2[0], (mem[2].field("h"), mem[2].field("wc"), mem[2].field("qz"))):
            np.testing.assert_array_equal(v, u)
    finally:
        batch.close()
        for m in mem:
            m.close()


def test_autotune_keeps_state_and_picks_options():
    cfgs = mix_configs()[:4]
    mem = [RichardsSolver(copy.deepcopy(c)) for c in cfgs]
    batch = RichardsBatch(mem)
    try:
        batch.step()
        before = [(m.field("h"), m.field("wc"), m.nextDt()) for m in mem]
        opts, best = batch.autotune(trials=1)
        assert opts["cells_per_block"] in (4096, 8192, 16384, 32768, 65536, 131072)
        assert best > 0.0
        for m, (h, wc, dt) in zip(mem, before):
            np.testing.assert_array_equal(m.field("h"), h)
            np.testing.assert_array_equal(m.field("wc"), wc)
            assert m.nextDt() == dt
        batch.step()
        assert batch.stats()["steps"] == 1
    finally:
        batch.close()
        for m in mem:
            m.close()
