"""Point decomposition over ranks, the reference's MPIBackend (ext/PartialFSHTMPIExt.jl:18-28).

Each rank holds a plan over its own points and replicated coefficients. Synthesis is local;
the adjoint of the global operator is the sum over ranks of the local adjoints, so it ends in
one all-reduce of the coefficient array (MPI.Allreduce! at ext/PartialFSHTMPIExt.jl:26; here
torch.distributed, NCCL between GPUs). As in the reference, a rank must be given only its
own points: passing the global set on every rank would scale the adjoint by the world size
(src/Plan.jl:64-67).

The plan may be any object with ``mul(f, alm)`` and ``mul_adjoint(alm, f)`` (a pfsht_b200
Plan on the rank's GPU in production).
"""
from __future__ import annotations

import numpy as np


def shard_points(theta, phi, rank: int, world: int):
    """Contiguous block of the points for `rank` (and its index range)."""
    n = len(theta)
    lo = (n * rank) // world
    hi = (n * (rank + 1)) // world
    return theta[lo:hi], phi[lo:hi], (lo, hi)


class PointShardedPlan:
    """mul! / mul!(', ...) of a plan whose points are split across the process group."""

    def __init__(self, local_plan, group=None):
        import torch.distributed as dist
        if not dist.is_initialized():
            raise RuntimeError("torch.distributed is not initialised")
        self.plan = local_plan
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)

    def mul(self, f, alm, **kw):
        """Local synthesis: f holds this rank's points (ext/PartialFSHTMPIExt.jl:18-20)."""
        return self.plan.mul(f, alm, **kw)

    def mul_adjoint(self, alm, f, **kw):
        """Local adjoint, then the sum over ranks (ext/PartialFSHTMPIExt.jl:22-28)."""
        import torch
        import torch.distributed as dist
        self.plan.mul_adjoint(alm, f, **kw)
        if isinstance(alm, np.ndarray):
            t = torch.from_numpy(alm)
            dist.all_reduce(torch.view_as_real(t), op=dist.ReduceOp.SUM, group=self.group)
            return alm
        if alm.is_cuda:
            torch.cuda.current_stream(alm.device).synchronize()
        dist.all_reduce(torch.view_as_real(alm), op=dist.ReduceOp.SUM, group=self.group)
        return alm
