"""GPU test of inqb_overlap_diagonal_noalloc, the entry point for callers that cannot let the
library allocate device memory (for example a serving loop whose memory is all handed to
resident orbital sets).  It must give the same per-state overlaps as inqb_overlap_diagonal,
call after call, while its partial sums live in a fixed array inside the library.

This file is collected last on purpose, so a run that stops at the first failure has already
run every other test."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-6


def _sets(ib, rng, sizes, nst, precision):
    rs = ib.RealSpace(ib.Cell.cubic(9.0), sizes=sizes)
    mk = lambda: rng.standard_normal(sizes + (nst,)) + 1j * rng.standard_normal(sizes + (nst,))
    return rs, ib.OrbitalSet.from_array(rs, mk(), precision=precision), ib.OrbitalSet.from_array(rs, mk(),
                                                                                                  precision=precision)


def _noalloc(ctx, a, b):
    """Call the entry point through the C ABI with a caller-owned device output buffer."""
    import torch
    out = torch.zeros(2 * a.nst, dtype=torch.float64, device="cuda")
    ctx.check(ctx.lib.inqb_overlap_diagonal_noalloc(a.handle, b.handle, C.c_void_p(out.data_ptr())))
    ctx.synchronize()
    v = out.cpu().numpy()
    return v[0::2] + 1j * v[1::2]


@pytest.mark.parametrize("precision_name", ["F64", "F32"])
def test_noalloc_matches_allocating_entry_point(precision_name, rng):
    import inq_b200 as ib
    prec = getattr(ib, precision_name)
    tol = TOL64 if prec == ib.F64 else TOL32
    rs, a, b = _sets(ib, rng, (24, 20, 18), 40, prec)
    rs2, c, d = _sets(ib, rng, (16, 16, 16), 200, prec)
    ctx = rs.ctx
    # two calls in a row with different shapes: the shared partial array is reused
    got1 = _noalloc(ctx, a, b)
    got2 = _noalloc(ctx, c, d)
    ref1 = ib.overlap_diagonal(a, b)
    ref2 = ib.overlap_diagonal(c, d)
    assert np.linalg.norm(got1 - ref1) / np.linalg.norm(ref1) < tol
    assert np.linalg.norm(got2 - ref2) / np.linalg.norm(ref2) < tol
    # and the first pair again after the larger one
    got3 = _noalloc(ctx, a, b)
    assert np.linalg.norm(got3 - ref1) / np.linalg.norm(ref1) < tol


def test_noalloc_rejects_oversize(rng):
    import inq_b200 as ib
    from inq_b200._lib import InqbError
    rs = ib.RealSpace(ib.Cell.cubic(5.0), sizes=(8, 8, 8))
    big = ib.OrbitalSet(rs, 513)
    big.fill(1.0)
    with pytest.raises(InqbError, match="at most 512 states"):
        _noalloc(rs.ctx, big, big)
