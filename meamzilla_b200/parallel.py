"""Several GPUs on one database: one process per GPU, the cells split.

The objective is a sum over cells (Potential::accumulate_error,
potential.cpp:415-491) plus the style punishment, so a database splits into
contiguous runs of cells, one per rank, balanced by triplet count as the
reference balances atoms over MPI ranks (AtomVec::init, atom_vec.cpp:41-140).
Each rank evaluates its cells for all candidates; one all-reduce (sum) of
[objective, gradient] per candidate over NCCL (gloo on CPU) completes the
step.  The punishment is counted on rank 0 only (omit_punishments on the
others).  Candidate populations can instead be split with no collective on the
data path (bench.py's weak-scaling mode).
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple

import numpy as np


def row_lengths_of_cells(cells, rcut: float) -> List[int]:
    """Work estimate per cell: triplets = sum over atoms of n(n-1)/2 with n the
    neighbour count, estimated as density * (4/3) pi rcut^3 (no lists built)."""
    out = []
    for c in cells:
        vol = abs(float(np.linalg.det(np.asarray(c.lattice, dtype=np.float64))))
        n = c.natoms / vol * 4.0 / 3.0 * np.pi * rcut ** 3
        out.append(int(c.natoms * n * max(n - 1.0, 0.0) / 2.0) + c.natoms)
    return out


def shard_cells(work: Sequence[float], world: int) -> List[Tuple[int, int]]:
    """Contiguous [lo, hi) cell ranges, one per rank, with near-equal work.
    Every rank gets at least one cell while there are enough cells."""
    work = np.asarray(work, dtype=np.float64)
    n = len(work)
    if world <= 0:
        raise ValueError("world must be positive")
    if n < world:
        raise ValueError("fewer cells (%d) than ranks (%d)" % (n, world))
    cum = np.concatenate([[0.0], np.cumsum(work)])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        k = int(np.searchsorted(cum, target))
        k = min(max(k, bounds[-1] + 1), n - (world - r))
        bounds.append(k)
    bounds.append(n)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


class ShardedObjective:
    """Objective (and gradient) of a database split over the ranks of a
    torch.distributed process group.

    `local(x) -> (obj[n], grad[n, P] or None)` evaluates this rank's cells for
    the candidate rows of x (on rank != 0 without the style punishment).
    The result is the sum over ranks, identical on every rank."""

    def __init__(self, local: Callable, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.local = local
        self.group = group
        if device is None and dist.get_backend(group) == "nccl":
            # NCCL reduces device buffers: this rank's current CUDA device
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = device

    def __call__(self, x, grad: bool = False):
        import torch
        x = np.atleast_2d(np.asarray(x, dtype=np.float64))
        obj, g = self.local(x, grad)
        n, P = x.shape
        buf = np.zeros(n * (1 + (P if grad else 0)))
        buf[:n] = obj
        if grad:
            buf[n:] = np.asarray(g).ravel()
        t = torch.tensor(buf, dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        out = t.cpu().numpy()
        if grad:
            return out[:n], out[n:].reshape(n, P)
        return out[:n]


def gpu_shard(cells, spec, rank: int, world: int, rcut: float, energy_weight=1.0, stress_weight=1.0,
              embed_extrap=0, max_candidates=1, device=None, make_evaluator=None):
    """This rank's evaluator for its run of cells: the GPU Evaluator, or
    whatever `make_evaluator` (same arguments as Evaluator) builds."""
    from .potential import Database, Evaluator, PotentialFile
    lo, hi = shard_cells(row_lengths_of_cells(cells, rcut), world)[rank]
    pot = PotentialFile.from_spec(spec)
    db = Database.from_cells(cells[lo:hi], pot)
    factory = Evaluator if make_evaluator is None else make_evaluator
    ev = factory(db, pot, energy_weight, stress_weight, embed_extrap, device=rank if device is None else device,
                 max_candidates=max_candidates, omit_punishments=(rank != 0))

    def local(x, grad):
        if grad:
            return ev.objective_grad(x)
        return ev.objective(x), None

    return ev, local, (lo, hi)
