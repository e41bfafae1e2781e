"""One domain over several ranks, on the host: the (i, j) slab partition,
the two-phase halo exchange and the distributed predictor solve, run as
gloo process groups of 2 and 4 ranks on 127.0.0.1 (no GPU).  The solve is
checked against the oracle's single-domain KSPCG on the same assembled
system: solution within 1e-9 relative, iteration count within +-2.  Also
the replica runs' aggregation bench.py does over ranks."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import dist_workers
from frehg_b200 import workloads
from frehg_b200.partition import SlabPartition, block_size, block_start, choose_grid

oracle = pytest.importorskip("oracle.gw")


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def spawn(fn, world, *args):
    mp.start_processes(fn, args=(world, free_port()) + args, nprocs=world, join=True,
                       start_method="spawn")


def test_block_rule_and_grid():
    assert [block_size(10, 3, r) for r in range(3)] == [4, 3, 3]
    assert [block_start(10, 3, r) for r in range(3)] == [0, 4, 7]
    assert choose_grid(64, 32, 8) == (4, 2)
    assert choose_grid(32, 64, 8) == (2, 4)
    assert choose_grid(1, 50, 4) == (1, 4)  # no empty blocks
    p = SlabPartition(10, 7, 5, 4)
    assert (p.px, p.py) == (2, 2)
    assert sum(b.nx * b.ny for b in p.blocks) == 70
    assert p.blocks[0].neighbor == (None, 1, None, 2)
    assert p.blocks[3].neighbor == (2, None, 1, None)
    g = np.random.default_rng(1).random((9, 12, 5))
    locs = [p.scatter(g, r) for r in range(4)]
    back = p.gather(locs)
    np.testing.assert_array_equal(back[1:-1, 1:-1], g[1:-1, 1:-1])


@pytest.mark.parametrize("world,grid", [(2, (2, 1)), (2, (1, 2)), (4, (2, 2))])
def test_halo_exchange(tmp_path, world, grid):
    shape = (9, 7, 6)
    spawn(dist_workers.halo_worker, world, shape, grid, str(tmp_path))
    part = SlabPartition(*shape, world, *grid)
    for r in range(world):
        z = np.load(tmp_path / f"halo{r}.npz")
        got, ref = z["got"], z["ref"]
        np.testing.assert_array_equal(got[1:-1, 1:-1], ref[1:-1, 1:-1])
        np.testing.assert_array_equal(z["got2"], 2.0 * got)
        e = part.edges(r)
        # halos facing a neighbour (corners included) hold its cells; the
        # domain-edge halos keep what they held
        rows = slice(0 if not e["south"] else 1, None if not e["north"] else -1)
        cols = slice(0 if not e["west"] else 1, None if not e["east"] else -1)
        np.testing.assert_array_equal(got[rows, cols], ref[rows, cols])
        if e["west"]:
            assert np.all(got[1:-1, 0] == -1.0)


def assembled_system(cfg, path):
    """The oracle's predictor system after one step, in the halo layout the
    B200 step stores it in (diag + upper legs, zero legs toward missing
    neighbours, identity rows outside the active cells), and the oracle's
    own KSPCG on it."""
    o = oracle.OracleSolver(cfg)
    dtg = o.next_dt()
    o.step(dtg, dtg)
    vals, cols, rhs = o.last_system()
    gid, _ = o.gid()
    nyh, nxh, nz = gid.shape
    diag = np.ones(gid.shape)
    gxp, gyp, gzp, b = (np.zeros(gid.shape) for _ in range(4))
    act = gid >= 0
    g = gid[act]
    diag[act] = vals[g, 0]
    gxp[act] = np.where(cols[g, 2] >= 0, vals[g, 2], 0.0)
    gyp[act] = np.where(cols[g, 4] >= 0, vals[g, 4], 0.0)
    gzp[act] = np.where(cols[g, 6] >= 0, vals[g, 6], 0.0)
    b[act] = rhs[g]
    s = cfg.solver
    x = np.zeros(len(rhs))
    res = C.c_double()
    lib = oracle.load()
    _dp = C.POINTER(C.c_double)
    its = lib.oracle_cg7(len(rhs), vals.ctypes.data_as(_dp),
                         cols.ctypes.data_as(C.POINTER(C.c_long)), rhs.ctypes.data_as(_dp),
                         x.ctypes.data_as(_dp), s.rtol, s.atol, s.max_iterations,
                         C.byref(res))
    xh = np.zeros(gid.shape)
    xh[act] = x[g]
    np.savez(path, diag=diag, gxp=gxp, gyp=gyp, gzp=gzp, b=b, rtol=s.rtol, atol=s.atol,
             maxit=s.max_iterations)
    o.close()
    return xh, its


@pytest.mark.parametrize("world,grid", [(2, (2, 1)), (2, (1, 2)), (4, (2, 2))])
def test_distributed_solve_matches_oracle(tmp_path, world, grid):
    cfg = workloads.hillslope(14, 11, 24)
    npz = str(tmp_path / "sys.npz")
    x_ref, its_ref = assembled_system(cfg, npz)
    assert its_ref > 20
    spawn(dist_workers.cg_worker, world, npz, grid, str(tmp_path))
    part = SlabPartition(14, 11, 24, world, *grid)
    outs = [np.load(tmp_path / f"cg{r}.npz") for r in range(world)]
    x = part.gather([o["x"] for o in outs])
    scale = max(float(np.max(np.abs(x_ref))), 1.0)
    assert float(np.max(np.abs(x - x_ref))) / scale <= 1e-9
    for o in outs:
        assert int(o["reason"]) > 0
        assert abs(int(o["its"]) - its_ref) <= 2
        assert int(o["its"]) == int(outs[0]["its"])
        assert float(o["dtmin"]) == 10.0
        assert float(o["tot"]) == sum(1.0 + r for r in range(world))


def test_replica_aggregation(tmp_path):
    spawn(dist_workers.replica_worker, 2, str(tmp_path))
    for r in range(2):
        z = np.load(tmp_path / f"rep{r}.npz")
        assert float(z["ms"]) == 110.0
        assert float(z["cells"]) == 3000.0
