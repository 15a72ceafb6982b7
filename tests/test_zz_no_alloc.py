"""GPU tests of inqb_overlap_diagonal_noalloc, the entry point for callers that cannot let the
library allocate device memory: a serving loop whose admission control has handed all device
memory to resident orbital sets, where a surprise cudaMalloc can fail or push out a request, and
latency-sensitive code that must not risk the implicit synchronisation of cudaMalloc/cudaFree.

It must give the per-state overlaps of the FP64 oracle (operations::overlap_diagonal,
src/operations/overlap_diagonal.hpp:25-55) call after call, make no device allocation (the
library's allocation counter and the device's free memory do not move across its calls, the
first ones on a fresh context included), and refuse output buffers a kernel must not store to.

This file is collected last on purpose, so a run that stops at the first failure has already
run every other test."""

import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-6


def _sets(ib, ctx, rng, sizes, nst, precision):
    lat = 9.0 * np.eye(3)
    rs = ib.RealSpace(ib.Cell(lat), sizes=sizes, ctx=ctx)
    mk = lambda: rng.standard_normal(sizes + (nst,)) + 1j * rng.standard_normal(sizes + (nst,))
    xa, xb = mk(), mk()
    a = ib.OrbitalSet.from_array(rs, xa, precision=precision)
    b = ib.OrbitalSet.from_array(rs, xb, precision=precision)
    # the oracle sees the values the device holds (rounded to complex64 for single precision)
    xa, xb = a.hypercubic().astype(np.complex128), b.hypercubic().astype(np.complex128)
    ors = O.RealSpace(O.Cell(lat), sizes)
    return a, b, O.overlap_diagonal(ors, xa, xb)


def _noalloc_raw(ctx, a, b, ptr):
    return ctx.lib.inqb_overlap_diagonal_noalloc(a.handle, b.handle, C.c_void_p(ptr))


def _as_complex(v):
    return v[0::2] + 1j * v[1::2]


@pytest.mark.parametrize("precision_name", ["F64", "F32"])
def test_noalloc_matches_oracle_and_allocates_nothing(precision_name, rng):
    import torch

    import inq_b200 as ib
    prec = getattr(ib, precision_name)
    tol = TOL64 if prec == ib.F64 else TOL32
    ctx = ib.Context(0)  # a fresh context: its first calls of the entry point are checked too
    try:
        a, b, ref1 = _sets(ib, ctx, rng, (24, 20, 18), 40, prec)
        c, d, ref2 = _sets(ib, ctx, rng, (16, 16, 16), 200, prec)
        # caller-owned outputs; the second starts one double into its buffer (8-byte aligned only)
        out1 = torch.zeros(2 * a.nst, dtype=torch.float64, device="cuda")
        out2 = torch.zeros(2 * c.nst + 1, dtype=torch.float64, device="cuda")
        out3 = torch.zeros(2 * a.nst, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        ctx.synchronize()
        allocs0 = ib.device_alloc_count()
        free0, _ = torch.cuda.mem_get_info()
        # two calls in a row with different shapes (the shared partial array is reused), then the first again
        ctx.check(_noalloc_raw(ctx, a, b, out1.data_ptr()))
        ctx.check(_noalloc_raw(ctx, c, d, out2.data_ptr() + 8))
        ctx.check(_noalloc_raw(ctx, a, b, out3.data_ptr()))
        ctx.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert ib.device_alloc_count() == allocs0
        assert free1 == free0
        got1 = _as_complex(out1.cpu().numpy())
        got2 = _as_complex(out2.cpu().numpy()[1:])
        got3 = _as_complex(out3.cpu().numpy())
        assert np.linalg.norm(got1 - ref1) / np.linalg.norm(ref1) < tol
        assert np.linalg.norm(got2 - ref2) / np.linalg.norm(ref2) < tol
        assert np.linalg.norm(got3 - ref1) / np.linalg.norm(ref1) < tol
        # and the allocating entry point agrees
        assert np.linalg.norm(ib.overlap_diagonal(a, b) - got1) / np.linalg.norm(ref1) < tol
        del a, b, c, d
    finally:
        ctx.synchronize()


def test_noalloc_refuses_bad_arguments(rng):
    import torch

    import inq_b200 as ib
    from inq_b200._lib import InqbError
    ctx = ib.Context.default()
    rs = ib.RealSpace(ib.Cell.cubic(5.0), sizes=(8, 8, 8))
    big = ib.OrbitalSet(rs, 513)
    big.fill(1.0)
    out = torch.zeros(2 * 513, dtype=torch.float64, device="cuda")
    with pytest.raises(InqbError, match="at most 512 states"):
        ctx.check(_noalloc_raw(ctx, big, big, out.data_ptr()))
    small = ib.OrbitalSet(rs, 4)
    small.fill(1.0)
    # host memory, pageable or page-locked, is refused before any kernel runs
    host = np.zeros(8)
    with pytest.raises(InqbError, match="device or managed memory"):
        ctx.check(_noalloc_raw(ctx, small, small, host.ctypes.data))
    pinned = torch.zeros(8, dtype=torch.float64).pin_memory()
    with pytest.raises(InqbError, match="device or managed memory"):
        ctx.check(_noalloc_raw(ctx, small, small, pinned.data_ptr()))
    with pytest.raises(InqbError, match="aligned"):
        ctx.check(_noalloc_raw(ctx, small, small, out.data_ptr() + 4))
    # the context is still usable
    ok = torch.zeros(8, dtype=torch.float64, device="cuda")
    ctx.check(_noalloc_raw(ctx, small, small, ok.data_ptr()))
    ctx.synchronize()
    np.testing.assert_allclose(_as_complex(ok.cpu().numpy()), np.full(4, rs.volume_element() * 512), rtol=1e-14)
