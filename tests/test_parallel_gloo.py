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
