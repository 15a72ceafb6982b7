"""States sharding on CPU ranks (gloo, world size 2): the partition follows the reference's
parallel::partition and the all-reduced per-rank densities equal the full density
(density.hpp:78-101), computed here with the oracle for each rank's block of states."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from inq_b200.parallel import Partition


def test_partition_matches_reference_rule():
    # partition.hpp:44-56: block = ceil(size / comm_size), start = min(block * rank, size)
    p = [Partition(10, 4, r) for r in range(4)]
    assert [(q.start, q.end) for q in p] == [(0, 3), (3, 6), (6, 9), (9, 10)]
    p = [Partition(3, 5, r) for r in range(5)]
    assert [q.local_size for q in p] == [1, 1, 1, 0, 0]
    assert sum(Partition(256, 8, r).local_size for r in range(8)) == 256


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    import oracle as O
    from inq_b200 import parallel
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        sizes, nst = (10, 12, 8), 7
        psi = rng.standard_normal(sizes + (nst,)) + 1j * rng.standard_normal(sizes + (nst,))
        occ = rng.uniform(0.5, 2.0, nst)
        part = Partition(nst, world, rank)
        local = O.density([psi[..., part.start:part.end]], [occ[part.start:part.end]])
        total = parallel.sharded_density(local)
        full = O.density([psi], [occ])
        out[rank] = float(np.max(np.abs(total - full)))
    finally:
        dist.destroy_process_group()


def test_sharded_density_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert len(out) == world
    assert max(out.values()) < 1e-13


class NumpyBlocks:
    """The block operations of the state-parallel algorithms on host arrays [nx][ny][nz][n] (the oracle's
    overlap, numpy products, gloo collectives), to check their bookkeeping on CPU ranks."""

    def __init__(self, rs, like):
        self.rs = rs
        self.like = like

    def empty(self, n):
        return np.zeros(self.like.shape[:-1] + (n,), np.complex128)

    def overlap(self, a, b):
        import oracle as O
        return O.overlap(self.rs, a, b)

    def multiply(self, a, R):
        npt = int(np.prod(a.shape[:-1]))
        return np.ascontiguousarray((a.reshape(npt, a.shape[-1]) @ R).reshape(a.shape[:-1] + (R.shape[1],)))

    def assign(self, dst, src):
        dst[...] = src

    def broadcast(self, blk, src):
        import torch
        import torch.distributed as dist
        dist.broadcast(torch.from_numpy(blk.view(np.float64)), src=src)
        return blk

    def reduce(self, blk, dst):
        import torch
        import torch.distributed as dist
        dist.reduce(torch.from_numpy(blk.view(np.float64)), dst=dst, op=dist.ReduceOp.SUM)
        return blk

    def allreduce(self, arr):
        from inq_b200 import parallel
        return np.ascontiguousarray(parallel.allreduce_sum(np.ascontiguousarray(arr).view(np.float64))).view(np.complex128)


def _blocks_main(rank, world, port, nst, out):
    import torch.distributed as dist
    import oracle as O
    from inq_b200 import parallel
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(9)
        rs = O.RealSpace(O.Cell(np.diag([5.0, 6.0, 4.5])), (6, 8, 5))
        sizes = rs.sizes
        psi = rng.standard_normal(sizes + (nst,)) + 1j * rng.standard_normal(sizes + (nst,))
        R = rng.standard_normal((nst, nst)) + 1j * rng.standard_normal((nst, nst))
        part = Partition(nst, world, rank)
        local = np.ascontiguousarray(psi[..., part.start:part.end])
        ops = NumpyBlocks(rs, local)
        S = parallel.sharded_overlap(local, part, blocks=ops)
        rot = parallel.sharded_rotate(local.copy(), R, part, blocks=ops)
        orth = parallel.sharded_orthogonalize(local.copy(), part, blocks=ops)
        V = 0.5 + np.cos(np.arange(int(np.prod(sizes))).reshape(sizes) / 7.0)
        sub = orth.copy()
        w = parallel.sharded_subspace_diagonalization(lambda x: V[..., None] * x, sub, part, blocks=ops)
        out[rank] = (part.start, part.end, S, rot, orth, w, sub)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nst", [(2, 7), (3, 7), (3, 2)])
def test_state_parallel_overlap_rotate_orthogonalize_gloo(world, nst):
    """overlap.hpp:42-56, rotate.hpp:27-62 and orthogonalize.hpp:25-31 over a state partition: every rank
    gets the full overlap, and the ranks' rotated and orthogonalised blocks put together equal the
    single-process results.  Ragged blocks (7 states over 2 or 3 ranks) and a rank without states (2
    states over 3 ranks)."""
    import oracle as O
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_blocks_main, args=(r, world, port, nst, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    rng = np.random.default_rng(9)
    rs = O.RealSpace(O.Cell(np.diag([5.0, 6.0, 4.5])), (6, 8, 5))
    psi = rng.standard_normal(rs.sizes + (nst,)) + 1j * rng.standard_normal(rs.sizes + (nst,))
    R = rng.standard_normal((nst, nst)) + 1j * rng.standard_normal((nst, nst))
    S_ref = O.overlap(rs, psi)
    rot = np.zeros_like(psi)
    orth = np.zeros_like(psi)
    sub = np.zeros_like(psi)
    for r in range(world):
        a, b, S, rr, oo, w, ss = out[r]
        assert np.max(np.abs(S - S_ref)) <= 1e-13 * np.max(np.abs(S_ref))
        rot[..., a:b] = rr
        orth[..., a:b] = oo
        sub[..., a:b] = ss
        if r == 0:
            w0 = w
        assert np.array_equal(w, w0)    # every rank forms the same eigenvalues
    rot_ref = (psi.reshape(-1, nst) @ R).reshape(psi.shape)
    assert np.max(np.abs(rot - rot_ref)) <= 1e-13 * np.max(np.abs(rot_ref))
    orth_ref = O.orthogonalize(rs, psi)
    assert np.max(np.abs(orth - orth_ref)) <= 1e-12 * np.max(np.abs(orth_ref))
    assert np.max(np.abs(O.overlap(rs, orth) - np.eye(nst))) < 1e-12
    # subspace diagonalisation of the orthonormal set under a real potential: <sub_i|V|sub_j> diagonal
    import inq_b200 as ib
    V = 0.5 + np.cos(np.arange(int(np.prod(rs.sizes))).reshape(rs.sizes) / 7.0)
    w_ref, U = ib.hermitian_eigen(O.overlap(rs, orth_ref, V[..., None] * orth_ref))
    assert np.max(np.abs(w0 - w_ref)) < 1e-12 * np.max(np.abs(w_ref))
    hs = O.overlap(rs, sub, V[..., None] * sub)
    assert np.max(np.abs(hs - np.diag(w_ref))) < 1e-11 * np.max(np.abs(w_ref))


def test_cholesky_inverse_host():
    """matrix::cholesky + invert_triangular (host FP64, no device needed): X = U^-1 with S = U^H U upper,
    and a matrix that is not positive definite is an error status."""
    import inq_b200 as ib
    from inq_b200 import _lib
    rng = np.random.default_rng(3)
    A = rng.standard_normal((9, 9)) + 1j * rng.standard_normal((9, 9))
    S = A.conj().T @ A + 0.5 * np.eye(9)
    X = ib.cholesky_inverse(S)
    U = np.linalg.cholesky(S).conj().T
    assert np.allclose(np.tril(X, -1), 0.0)
    assert np.max(np.abs(X - np.linalg.inv(U))) < 1e-12 * np.max(np.abs(X))
    assert np.max(np.abs(X.conj().T @ S @ X - np.eye(9))) < 1e-12
    with pytest.raises(_lib.InqbError):
        ib.cholesky_inverse(-np.eye(3))
