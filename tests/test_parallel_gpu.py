"""GPU tests of the state-parallel overlap, rotation, orthogonalisation, subspace diagonalisation and
ETRS step (overlap.hpp:42-56, rotate.hpp:27-142, orthogonalize.hpp:25-31, subspace_diagonalization.hpp:21-29,
density.hpp:99) through the device kernels.

One GPU is available per run, so: the rectangular rotation kernel against numpy; the NCCL path (device
buffers viewed in place, collectives ordered on the context's stream) with one rank; and two ranks as
processes on the same GPU exchanging blocks through host memory over gloo (their kernels never wait
on one another).  Results: equal to the single-set operations to 1e-12."""

import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _system(nst, seed=21):
    import inq_b200 as ib
    rs = ib.RealSpace(ib.Cell(np.diag([7.0, 6.5, 7.5])), sizes=(20, 18, 24))
    rng = np.random.default_rng(seed)
    psi = rng.standard_normal(rs.sizes + (nst,)) + 1j * rng.standard_normal(rs.sizes + (nst,))
    return rs, psi


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_rotate_to_rectangular(precision):
    import inq_b200 as ib
    rs, psi = _system(12)
    prec = ib.F64 if precision == "f64" else ib.F32
    rng = np.random.default_rng(4)
    phi = ib.OrbitalSet.from_array(rs, psi, precision=prec)
    R = rng.standard_normal((12, 5)) + 1j * rng.standard_normal((12, 5))
    y0 = rng.standard_normal(rs.sizes + (5,)) + 1j * rng.standard_normal(rs.sizes + (5,))
    out = ib.OrbitalSet.from_array(rs, y0, precision=prec)
    alpha, beta = 0.7 - 0.2j, -0.3 + 1.1j
    ib.rotate_to(phi, out, R, alpha, beta)
    x = phi.matrix().astype(np.complex128)
    ref = alpha * (x @ R) + beta * y0.reshape(-1, 5).astype(np.complex64 if prec == ib.F32 else np.complex128)
    tol = 1e-13 if prec == ib.F64 else 2e-6
    assert np.max(np.abs(out.matrix() - ref)) <= tol * np.max(np.abs(ref))
    # alpha = 1, beta = 0: plain product into a fresh set, the in-place rotation's arithmetic
    sq = rng.standard_normal((12, 12)) + 1j * rng.standard_normal((12, 12))
    a = ib.rotate_to(phi, phi.skeleton(), sq).matrix()
    b = ib.rotate(phi.copy(), sq).matrix()
    assert np.array_equal(a, b)


def test_state_parallel_nccl_one_rank():
    import torch
    import torch.distributed as dist
    import inq_b200 as ib
    from inq_b200 import parallel
    rs, psi = _system(10)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1)
    try:
        part = parallel.Partition(10, 1, 0)
        phi = ib.OrbitalSet.from_array(rs, psi)
        S = parallel.sharded_overlap(phi, part)
        assert np.max(np.abs(S - ib.overlap(phi))) <= 1e-14 * np.max(np.abs(S))
        ref = ib.orthogonalize(phi.copy()).matrix()
        got = parallel.sharded_orthogonalize(phi, part).matrix()
        assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))
        ham = _hamiltonian(rs)
        single = phi.copy()
        w_ref = ham.subspace_diagonalization(single)
        w = parallel.sharded_subspace_diagonalization(ham, phi, part)
        assert np.max(np.abs(w - w_ref)) <= 1e-13 * np.max(np.abs(w_ref))
        assert np.max(np.abs(phi.matrix() - single.matrix())) <= 1e-12 * np.max(np.abs(single.matrix()))
        # the state-sharded ETRS step: the density stays on the device and is all-reduced there
        occ = np.full(10, 2.0)
        a, b = phi.copy(), phi.copy()
        dens, dip, it = parallel.sharded_etrs_step(ham, a, occ, 0.01, rs)
        assert isinstance(dens, torch.Tensor) and dens.is_cuda
        dref, dipref, itref = ib.etrs(ham, [b], [occ], 0.01, want_density=True)
        assert it == itref
        assert np.array_equal(dens.cpu().numpy(), dref)
        assert np.max(np.abs(dip - dipref)) <= 1e-13 * np.max(np.abs(dipref))
        assert np.array_equal(a.matrix(), b.matrix())
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()


def _hamiltonian(rs):
    import inq_b200 as ib
    ham = ib.KSHamiltonian(rs)
    n = int(np.prod(rs.sizes))
    ham.set_scalar_potential((0.4 + 0.3 * np.cos(np.arange(n) / 11.0)).reshape(rs.sizes))
    return ham


def _rank_main(rank, world, port, nst, out):
    import torch.distributed as dist
    import inq_b200 as ib
    from inq_b200 import parallel
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rs, psi = _system(nst)
        part = parallel.Partition(nst, world, rank)
        phi = ib.OrbitalSet.from_array(rs, psi[..., part.start:part.end])
        S = parallel.sharded_overlap(phi, part)
        parallel.sharded_orthogonalize(phi, part)
        orth = phi.hypercubic()
        w = parallel.sharded_subspace_diagonalization(_hamiltonian(rs), phi, part)
        # the state-sharded ETRS step over gloo (host arrays): global density and dipole on every rank
        occ = np.linspace(0.5, 2.0, nst)[part.start:part.end]
        p2 = ib.OrbitalSet.from_array(rs, psi[..., part.start:part.end])
        dens, dip, _ = parallel.sharded_etrs_step(_hamiltonian(rs), p2, occ, 0.01, rs)
        out[rank] = (part.start, part.end, S, orth, w, phi.hypercubic(), dens, dip)
    finally:
        dist.destroy_process_group()


def test_state_parallel_two_ranks_one_gpu():
    import torch.multiprocessing as mp
    import inq_b200 as ib
    nst, world = 13, 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, nst, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    rs, psi = _system(nst)
    phi = ib.OrbitalSet.from_array(rs, psi)
    S_ref = ib.overlap(phi)
    ref = ib.orthogonalize(phi).hypercubic()
    ham = _hamiltonian(rs)
    w_ref = ham.subspace_diagonalization(phi)
    got = np.zeros_like(ref)
    sub = np.zeros_like(ref)
    single = ib.OrbitalSet.from_array(rs, psi)
    dref, dipref, _ = ib.etrs(ham, [single], [np.linspace(0.5, 2.0, nst)], 0.01, want_density=True)
    for r in range(world):
        a, b, S, blk, w, sb, dens, dip = out[r]
        assert np.max(np.abs(dens - dref)) <= 1e-12 * np.max(np.abs(dref))
        assert np.max(np.abs(dip - dipref)) <= 1e-11 * np.max(np.abs(dipref))
        assert np.max(np.abs(S - S_ref)) <= 1e-13 * np.max(np.abs(S_ref))
        assert np.max(np.abs(w - w_ref)) <= 1e-12 * np.max(np.abs(w_ref))
        got[..., a:b] = blk
        sub[..., a:b] = sb
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert np.max(np.abs(ib.overlap(ib.OrbitalSet.from_array(rs, got)) - np.eye(nst))) < 1e-12
    # the rotated states diagonalise the subspace Hamiltonian like the single-set call
    sub_set = ib.OrbitalSet.from_array(rs, sub)
    hs = ib.overlap(sub_set, ham(sub_set))
    assert np.max(np.abs(hs - np.diag(w_ref))) <= 1e-11 * np.max(np.abs(w_ref))
    assert np.max(np.abs(sub - phi.hypercubic())) <= 1e-10 * np.max(np.abs(sub))
