"""Rank bodies of the multi-process CPU tests (gloo, 127.0.0.1): spawned
processes import them from here."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _init(rank, world, port):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    return dist


def halo_worker(rank, world, port, shape, grid, out_dir):
    """Owned cells from a known global field, halos poisoned; after the
    exchange every halo cell facing a neighbour holds the global value."""
    import torch

    from frehg_b200.partition import HaloExchange, SlabPartition
    dist = _init(rank, world, port)
    try:
        nx, ny, nz = shape
        part = SlabPartition(nx, ny, nz, world, *grid)
        g = np.arange((ny + 2) * (nx + 2) * nz, dtype=np.float64).reshape(ny + 2, nx + 2, nz)
        loc = part.scatter(g, rank).copy()
        ref = loc.copy()
        loc[0, :] = -1.0
        loc[-1, :] = -1.0
        loc[:, 0] = -1.0
        loc[:, -1] = -1.0
        a = torch.from_numpy(loc)
        b = torch.from_numpy(2.0 * loc)
        HaloExchange(part, rank, dist).exchange([a, b])
        np.savez(os.path.join(out_dir, f"halo{rank}.npz"), got=a.numpy(), got2=b.numpy(), ref=ref)
    finally:
        dist.destroy_process_group()


def cg_worker(rank, world, port, npz, grid, out_dir):
    """The distributed KSPCG on this rank's block of the saved system."""
    import torch

    from frehg_b200 import dcg
    from frehg_b200.partition import SlabPartition
    dist = _init(rank, world, port)
    try:
        z = np.load(npz)
        ny, nx, nz = z["diag"].shape[0] - 2, z["diag"].shape[1] - 2, z["diag"].shape[2]
        part = SlabPartition(nx, ny, nz, world, *grid)
        t = {k: torch.from_numpy(part.scatter(z[k], rank)) for k in ("diag", "gxp", "gyp", "gzp", "b")}
        b = t["b"].clone()
        b[0, :] = 0.0
        b[-1, :] = 0.0
        b[:, 0] = 0.0
        b[:, -1] = 0.0
        # only the owned rows' legs are this rank's; the halo legs arrive
        # from the neighbours (domain-edge halos stay 0)
        for k in ("gxp", "gyp"):
            t[k][0, :] = 0.0
            t[k][-1, :] = 0.0
            t[k][:, 0] = 0.0
            t[k][:, -1] = 0.0
        sys_ = dcg.LocalSystem(part, rank, t["diag"], t["gxp"], t["gyp"], t["gzp"], b, dist)
        sys_.share_legs()
        x, info = dcg.solve(sys_, rtol=float(z["rtol"]), atol=float(z["atol"]),
                            maxit=int(z["maxit"]))
        dtmin = dcg.global_min(dist, 10.0 + rank)
        tot = dcg.global_sum(dist, 1.0 + rank)
        np.savez(os.path.join(out_dir, f"cg{rank}.npz"), x=x.numpy(), its=info.iterations,
                 reason=info.reason, dtmin=dtmin, tot=tot)
    finally:
        dist.destroy_process_group()


def replica_worker(rank, world, port, out_dir):
    """bench.py's aggregation of a replica run: the slowest rank's time and
    the cells of all ranks."""
    import bench
    dist = _init(rank, world, port)
    try:
        ms, cells = bench.reduce_over_ranks(dist, 100.0 + 10.0 * rank, 1000 * (rank + 1), "cpu")
        np.savez(os.path.join(out_dir, f"rep{rank}.npz"), ms=ms, cells=cells)
    finally:
        dist.destroy_process_group()
