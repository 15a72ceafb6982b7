"""States sharding over ranks (one process per GPU).

The Kohn-Sham operator has no exchange between states, so orbitals split over ranks
like INQ's state partition (basis/field_set.hpp:58-74 with parallel/partition.hpp:25-60):
every rank applies H and propagates its own block of states, and the only collective of
a propagation is the sum of the per-rank densities (density.hpp:99) and of the scalar
observables built on them.  The operations that couple states exchange blocks of them:
the overlap matrix (overlap.hpp:42-56: every rank's block reaches every rank, then an
all-reduce of the S x S matrix), the rotation (rotate.hpp:27-62: each rank's products
for a destination block are summed on its owner) and the orthogonalisation built from
both.  The collectives go through ``torch.distributed``: NCCL on the device buffers
between GPUs, or any other backend through host copies.  No TMA multicast or peer memory
is involved.
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

    With the fixed Hamiltonian of the synthetic configurations the states evolve independently, so the
    only exchanges are the density sum (density.hpp:99) and the sum of the dipoles, which are linear in
    the density.  With NCCL the step writes its density into a device tensor and the all-reduce runs on
    it in place: the density never leaves the device (returned as that tensor).  Other backends add
    host arrays."""
    import torch
    import torch.distributed as dist
    from . import core
    nccl = dist.is_initialized() and dist.get_backend(group) == "nccl"
    if nccl:
        dev = torch.device("cuda", ham.ctx.device)
        dens = torch.empty(basis.size(), dtype=torch.float64, device=dev)
        _, dip, iters = core.etrs(ham, [phi_local], [occ_local], dt, density_out=dens)
        dipt = torch.as_tensor(dip, dtype=torch.float64, device=dev)
        # the step returned after its stream finished, so the tensors are complete for the collective
        dist.all_reduce(dens, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(dipt, op=dist.ReduceOp.SUM, group=group)
        return dens, dipt.cpu().numpy(), iters
    dens_local, dip_local, iters = core.etrs(ham, [phi_local], [occ_local], dt, want_density=True)
    dens = sharded_density(dens_local, group, device)
    return dens, allreduce_sum(dip_local, group, device), iters


class _DeviceWords:
    """A raw device buffer as a 1-D array of float64 or float32 words (__cuda_array_interface__), so
    that ``torch.as_tensor`` views it without a copy."""

    def __init__(self, ptr: int, nwords: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (nwords,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


class SetBlocks:
    """Block operations of the state-parallel algorithms on orbital sets of this rank.

    Blocks are ``OrbitalSet`` objects on the rank's context; their products run on the device.  With
    the NCCL backend the collectives read and write the sets' device memory in place, ordered on the
    context's stream; with any other backend a block travels through host memory."""

    def __init__(self, like, group=None):
        import torch.distributed as dist
        self.like = like
        self.group = group
        self.nccl = dist.is_initialized() and dist.get_backend(group) == "nccl"

    # -- products (device)
    def empty(self, nst: int):
        from .core import OrbitalSet
        p = self.like
        return OrbitalSet(p.basis, nst, 1, p._kpoint, p._spin, p.space, p.precision)

    def overlap(self, a, b) -> np.ndarray:
        from .core import overlap
        return overlap(a, b)

    def multiply(self, a, R: np.ndarray):
        from .core import rotate_to
        out = self.empty(R.shape[1])
        return rotate_to(a, out, R)

    def assign(self, dst, src):
        dst.assign(src)

    # -- collectives
    def _tensor(self, blk):
        import torch
        words = blk.basis.size() * blk.nst * 2
        typestr = "<f8" if blk.dtype == np.complex128 else "<f4"
        return torch.as_tensor(_DeviceWords(blk.device_ptr(), words, typestr), device=f"cuda:{blk.ctx.device}")

    def _collective(self, blk, fn):
        import torch
        if self.nccl:
            with torch.cuda.stream(torch.cuda.ExternalStream(blk.ctx.stream(), device=f"cuda:{blk.ctx.device}")):
                fn(self._tensor(blk))
            return blk
        host = blk.matrix()
        t = torch.from_numpy(np.ascontiguousarray(host).view(np.float64 if host.dtype == np.complex128 else np.float32))
        fn(t)
        blk.upload(t.numpy().view(host.dtype).reshape(host.shape))
        return blk

    def broadcast(self, blk, src: int):
        import torch.distributed as dist
        return self._collective(blk, lambda t: dist.broadcast(t, src=src, group=self.group))

    def reduce(self, blk, dst: int):
        import torch.distributed as dist
        return self._collective(blk, lambda t: dist.reduce(t, dst=dst, op=dist.ReduceOp.SUM, group=self.group))

    def allreduce(self, arr: np.ndarray) -> np.ndarray:
        out = allreduce_sum(np.ascontiguousarray(arr).view(np.float64), self.group,
                            f"cuda:{self.like.ctx.device}" if self.nccl else None)
        return np.ascontiguousarray(out).view(np.complex128)


def sharded_overlap(phi1, part: Partition, phi2=None, group=None, blocks=None) -> np.ndarray:
    """operations::overlap of state-partitioned sets (overlap.hpp:42-56): the full S x S matrix
    <phi1_i|phi2_j> on every rank.

    Every rank's block of ``phi1`` is broadcast in turn; each rank fills the columns of its own
    ``phi2`` states against it, and a sum over ranks (each column written by exactly one) completes
    the matrix.  ``part`` is this rank's partition of the S states; ``phi2`` defaults to ``phi1``."""
    ops = blocks or SetBlocks(phi1, group)
    phi2 = phi1 if phi2 is None else phi2
    S = part.size
    out = np.zeros((S, S), np.complex128)
    for ip in range(part.comm_size):
        pi = Partition(S, part.comm_size, ip)
        if pi.local_size == 0:
            continue
        blk = phi1 if ip == part.rank else ops.empty(pi.local_size)
        blk = ops.broadcast(blk, ip)
        if part.local_size:
            out[pi.start:pi.end, part.start:part.end] = ops.overlap(blk, phi2)
    return ops.allreduce(out)


def sharded_rotate(phi, R, part: Partition, group=None, blocks=None):
    """operations::rotate of a state-partitioned set (rotate.hpp:27-62): phi <- phi R with the full
    [S][S] matrix R on every rank.

    For each destination block every rank multiplies its local states by its rows of that block's
    columns of R; the products are summed on the block's owner, which takes the sum as its new states
    once all blocks are done."""
    ops = blocks or SetBlocks(phi, group)
    R = np.asarray(R, dtype=np.complex128)
    S = part.size
    result = None
    for ip in range(part.comm_size):
        pi = Partition(S, part.comm_size, ip)
        if pi.local_size == 0:
            continue
        blk = ops.multiply(phi, R[part.start:part.end, pi.start:pi.end])
        blk = ops.reduce(blk, ip)
        if ip == part.rank:
            result = blk
    if result is not None:
        ops.assign(phi, result)
    return phi


def sharded_orthogonalize(phi, part: Partition, group=None, blocks=None):
    """operations::orthogonalize of a state-partitioned set (orthogonalize.hpp:25-31): the all-reduced
    overlap, its Cholesky inverse formed in FP64 on every rank (the same matrix on all of them), and the
    state-parallel rotation."""
    from .core import cholesky_inverse
    ops = blocks or SetBlocks(phi, group)
    S = sharded_overlap(phi, part, None, group, ops)
    return sharded_rotate(phi, cholesky_inverse(S), part, group, ops)


def sharded_subspace_diagonalization(ham, phi, part: Partition, group=None, blocks=None) -> np.ndarray:
    """ground_state::subspace_diagonalization of a state-partitioned set (subspace_diagonalization.hpp:21-29):
    H applied to the local states (it couples none), the all-reduced <phi_i|H phi_j>, its eigenvectors
    formed in FP64 on every rank and the state-parallel rotation onto them.  Returns the eigenvalues."""
    from .core import hermitian_eigen
    ops = blocks or SetBlocks(phi, group)
    hs = sharded_overlap(phi, part, ham(phi), group, ops)
    w, V = hermitian_eigen(hs)
    sharded_rotate(phi, V, part, group, ops)
    return w
