"""The predictor solve of one domain split over several ranks.

The reference's head system is a PETSc MPIAIJ matrix whose rows each rank
owns by its (i, j) block (``src/core/LinearSystem.cpp:147-151, 311-484``);
every CG iteration exchanges the direction vector's one-cell halo and
all-reduces the dot products.  :func:`solve` restates that KSPCG (x0 = 0,
Hestenes-Stiefel, preconditioned norm, the reference's rtol / atol / maxit
and divergence tests; the Jacobi lane ``-gw_pc_type jacobi``) on the
matrix-free 7-point form the B200 step stores -- the diagonal and the three
upper legs of every cell in the local halo layout ``(ny + 2, nx + 2, nz)``,
legs toward a missing neighbour 0 -- with the halo exchange of
:class:`frehg_b200.partition.HaloExchange` and ``all_reduce`` sums, so it
runs over NCCL with CUDA tensors and over gloo with CPU tensors.

:func:`global_min` and :func:`global_sum` are the step's other collectives:
the controller's dt MIN (``src/gw/AdaptiveStep.cpp:115-116``) and the audit
sums.
"""
from __future__ import annotations

from dataclasses import dataclass

from .partition import HaloExchange, SlabPartition

# KSPConvergedReason values the reference reads (LinearSystem.cpp:426-431)
CONVERGED_RTOL, CONVERGED_ATOL = 2, 3
DIVERGED_ITS, DIVERGED_DTOL, DIVERGED_NANORINF = -3, -4, -9
DIVERGED_INDEFINITE_PC, DIVERGED_INDEFINITE_MAT = -8, -10


@dataclass
class SolveInfo:
    iterations: int
    residual: float  # final preconditioned norm ||D^-1 r||
    reason: int


def global_sum(dist, value, group=None):
    """Sum over ranks of a tensor (in place) or a float."""
    import torch
    t = value if torch.is_tensor(value) else torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t if torch.is_tensor(value) else float(t.item())


def global_min(dist, value: float, device=None, group=None) -> float:
    """The minimum over ranks (the controller's next dt)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    return float(t.item())


class LocalSystem:
    """One rank's rows: diag, gxp, gyp, gzp and b in the local halo layout
    (torch tensors, one device).  The legs' west / south halos are the
    neighbours' upper legs toward this block (filled by :meth:`share_legs`);
    at the domain's edges they stay 0."""

    def __init__(self, part: SlabPartition, rank: int, diag, gxp, gyp, gzp, b, dist,
                 group=None):
        self.part, self.rank, self.dist, self.group = part, rank, dist, group
        self.diag, self.gxp, self.gyp, self.gzp, self.b = diag, gxp, gyp, gzp, b
        self.halo = HaloExchange(part, rank, dist, group)
        self.inner = (slice(1, -1), slice(1, -1))

    def share_legs(self) -> None:
        self.halo.exchange([self.gxp, self.gyp])

    def apply(self, p, out) -> None:
        """out = A p on the owned cells (p's halo current), in the SpMV's
        order ym, xm, zm, diag, zp, xp, yp."""
        P = p
        J, I = self.inner
        c = P[J, I]
        y = self.gyp[0:-2, 1:-1] * P[0:-2, 1:-1]
        y = y + self.gxp[1:-1, 0:-2] * P[1:-1, 0:-2]
        zm = self.gzp[J, I].new_zeros(c.shape)
        zm[..., 1:] = self.gzp[J, I][..., :-1] * c[..., :-1]
        y = y + zm
        y = y + self.diag[J, I] * c
        zp = self.gzp[J, I].new_zeros(c.shape)
        zp[..., :-1] = self.gzp[J, I][..., :-1] * c[..., 1:]
        y = y + zp
        y = y + self.gxp[J, I] * P[1:-1, 2:]
        y = y + self.gyp[J, I] * P[2:, 1:-1]
        out[J, I] = y

    def dot(self, u, v) -> float:
        J, I = self.inner
        s = (u[J, I] * v[J, I]).sum().reshape(1)
        return float(global_sum(self.dist, s, self.group).item())


def solve(sys_: LocalSystem, rtol: float = 1e-8, atol: float = 1e-14, maxit: int = 1000,
          dtol: float = 1e5):
    """KSPCG with Jacobi on the distributed system; returns (x, SolveInfo).
    x is the local halo-layout solution (ring 0)."""
    import math

    import torch
    J, I = sys_.inner
    b = sys_.b
    dinv = torch.where(sys_.diag != 0, 1.0 / sys_.diag, torch.ones_like(sys_.diag))
    x = torch.zeros_like(b)
    r = b.clone()
    z = torch.zeros_like(b)
    p = torch.zeros_like(b)
    w = torch.zeros_like(b)
    z[J, I] = r[J, I] * dinv[J, I]
    dp = math.sqrt(sys_.dot(z, z))
    rnorm0 = dp
    ttol = max(rtol * rnorm0, atol)
    reason = 0

    def test(rn):
        if not math.isfinite(rn):
            return DIVERGED_NANORINF
        if rn <= ttol:
            return CONVERGED_ATOL if rn < atol else CONVERGED_RTOL
        if rn >= dtol * rnorm0:
            return DIVERGED_DTOL
        return 0

    reason = test(dp)
    its = 0
    if reason == 0:
        beta, betaold, dpi, dpiold = sys_.dot(z, r), 1.0, 0.0, 0.0
        i = 0
        while True:
            its = i + 1
            if beta == 0.0:
                reason = CONVERGED_ATOL
                break
            if i > 0 and beta * betaold < 0.0:
                reason = DIVERGED_INDEFINITE_PC
                break
            if i == 0:
                p[J, I] = z[J, I]
            else:
                p[J, I] = z[J, I] + (beta / betaold) * p[J, I]
            sys_.halo.exchange([p])
            dpiold = dpi
            sys_.apply(p, w)
            dpi = sys_.dot(p, w)
            betaold = beta
            if dpi == 0.0 or (i > 0 and math.copysign(1.0, dpi) != math.copysign(1.0, dpiold)):
                reason = DIVERGED_INDEFINITE_MAT
                break
            a = beta / dpi
            x[J, I] += a * p[J, I]
            r[J, I] -= a * w[J, I]
            z[J, I] = r[J, I] * dinv[J, I]
            dp = math.sqrt(sys_.dot(z, z))
            reason = test(dp)
            if reason != 0:
                break
            beta = sys_.dot(z, r)
            i += 1
            if i >= maxit:
                reason = DIVERGED_ITS
                break
    return x, SolveInfo(its, dp, reason)
