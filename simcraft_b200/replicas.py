"""Replica plumbing for runs with one process per GPU.

The FluidSim path does not shard: the MIC(0) sweeps are one global i+j+k
wavefront, so N GPUs run N independent replicas (one solve or scene each) and
meet only on the host side of the measurement:

  Replicas.from_env()            rank / world from torchrun's environment
  replicas.max(x)                max over ranks (the slowest replica's time)
  replicas.shard(n)              round-robin share of n independent work items
  replicas.gather(obj)           every rank's object, in rank order, on all ranks
  fd_check(...)                  central differences along seeded directions,
                                 the directions split round-robin over ranks

With world == 1 every call is local and no process group is needed.
"""
import os

import numpy as np


class Replicas:
    def __init__(self, rank=0, world=1, dist=None, device=None):
        self.rank, self.world, self.dist = int(rank), int(world), dist
        self.device = device  # tensor device of the collectives ("cpu" for gloo)

    @classmethod
    def from_env(cls, dist=None, device=None):
        return cls(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), dist, device)

    @property
    def active(self):
        return self.dist is not None and self.world > 1

    def barrier(self):
        if self.active:
            self.dist.barrier()

    def max(self, value):
        """Maximum of a float over ranks."""
        if not self.active:
            return float(value)
        import torch

        t = torch.tensor([float(value)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def shard(self, n):
        """Indices of the work items this rank takes: i = rank, rank + world, ..."""
        return list(range(self.rank, int(n), self.world))

    def gather(self, obj):
        """[obj of rank 0, obj of rank 1, ...] on every rank."""
        if not self.active:
            return [obj]
        out = [None] * self.world
        self.dist.all_gather_object(out, obj)
        return out

    def unshard(self, n, parts):
        """Reassemble per-rank lists of shard() results into item order."""
        items = [None] * int(n)
        for r, part in enumerate(parts):
            for i, v in zip(range(r, int(n), self.world), part):
                items[i] = v
        return items


def fd_directions(shape, count, seed):
    """The seeded directions of the finite-difference check, in order (every
    rank draws all of them, so the k-th direction does not depend on the
    number of ranks)."""
    rng = np.random.default_rng(seed)
    return [rng.standard_normal(shape) for _ in range(count)]


def fd_check(loss_at, grad_dot, shape, count, seed, eps, replicas=None):
    """Relative errors |fd - ad| / max(|fd|, |ad|) of the adjoint along `count`
    seeded directions, fd = (L(U + eps d) - L(U - eps d)) / (2 eps) and
    ad = <grad, d>.  `loss_at(d, sign)` evaluates L(U + sign*eps*d) and
    `grad_dot(d)` returns <grad, d>.  Each rank evaluates its round-robin share;
    the result (all directions, in order) is returned on every rank."""
    replicas = replicas or Replicas()
    dirs = fd_directions(shape, count, seed)
    mine = []
    for i in replicas.shard(count):
        d = dirs[i]
        fd = (loss_at(d, +1.0) - loss_at(d, -1.0)) / (2.0 * eps)
        ad = grad_dot(d)
        mine.append(abs(fd - ad) / max(abs(fd), abs(ad), 1e-300))
    return replicas.unshard(count, replicas.gather(mine))


__all__ = ["Replicas", "fd_directions", "fd_check"]
