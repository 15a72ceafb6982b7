"""States sharding over ranks (one process per GPU).

The Kohn-Sham operator has no exchange between states, so orbitals split over ranks
like INQ's state partition (basis/field_set.hpp:58-74 with parallel/partition.hpp:25-60):
every rank applies H and propagates its own block of states, and the only collective is
the sum of the per-rank densities (density.hpp:99) and of the scalar observables built on
them.  The collectives go through ``torch.distributed``: NCCL between GPUs, gloo on CPU
(tests).  No TMA multicast or peer memory is involved.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Partition:
    """Block partition of ``size`` items over ``comm_size`` ranks (parallel::partition)."""
    size: int
    comm_size: int
    rank: int

    @property
    def block(self) -> int:
        return (self.size + self.comm_size - 1) // self.comm_size

    @property
    def start(self) -> int:
        return min(self.block * self.rank, self.size)

    @property
    def end(self) -> int:
        return min(self.block * (self.rank + 1), self.size)

    @property
    def local_size(self) -> int:
        return self.end - self.start

    def local_to_global(self, i: int) -> int:
        return self.start + i


def allreduce_sum(array: np.ndarray, group=None, device=None) -> np.ndarray:
    """Sum a float64 array over the ranks of ``group`` (in place semantics of all_reduce_in_place_n)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return array
    t = torch.from_numpy(np.ascontiguousarray(array, dtype=np.float64))
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def sharded_density(local_density: np.ndarray, group=None, device=None) -> np.ndarray:
    """density::calculate over all ranks: each rank's sum over its states, added over ranks."""
    return allreduce_sum(local_density, group, device)


def sharded_etrs_step(ham, phi_local, occ_local, dt: float, basis, group=None, device=None):
    """One ETRS step on this rank's block of states, then the global density and dipole.

    With the fixed Hamiltonian of the synthetic configurations the states evolve
    independently, so the only exchange is the density sum."""
    from . import core
    dens_local, _, iters = core.etrs(ham, [phi_local], [occ_local], dt, want_density=True)
    dens = sharded_density(dens_local, group, device)
    return dens, core.dipole(basis, dens), iters
