"""GPU tests of inqb_apply_host, ks_hamiltonian::operator() on a set held in host memory.

The states stream through the device in blocks, with the uploads and downloads overlapping the
operator.  The result must match the device-resident call (upload, inqb_apply, download) within
the parity tolerances of the other tests: 1e-12 relative for double precision, 2e-6 for single.
Block sizes cover one block, several blocks with a ragged last one, and the default; the host
arrays are both pageable (numpy) and page-locked."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    import inq_b200 as ib
    from inq_b200 import synthetic
    sysm = synthetic.config("c1", nst=40)
    basis, ham, phi = synthetic.build(sysm)
    return ib, basis, ham, phi


@pytest.mark.parametrize("precision_name,tol", [("F64", 1e-12), ("F32", 2e-6)])
@pytest.mark.parametrize("block", [0, 16, 40])
def test_apply_host_matches_device_call(c1, precision_name, tol, block):
    ib, basis, ham, phi64 = c1
    prec = getattr(ib, precision_name)
    phi = phi64 if prec == ib.F64 else phi64.converted(prec)
    ref = ham(phi).matrix()
    host_in = np.ascontiguousarray(phi.matrix())
    host_out = np.zeros_like(host_in)
    ham.apply_host(host_in, host_out, block_states=block)
    err = np.linalg.norm(host_out - ref) / np.linalg.norm(ref)
    assert err < tol, err


@pytest.mark.parametrize("precision_name,tol", [("F64", 1e-12), ("F32", 2e-6)])
def test_apply_host_default_blocks_ragged_end(precision_name, tol):
    """136 states with the default blocks: full blocks and a short last one (single: 64, 64, 8;
    double: 32, 32, 32, 32, 8)."""
    import inq_b200 as ib
    from inq_b200 import synthetic
    sysm = synthetic.config("c1", nst=136)
    basis, ham, phi64 = synthetic.build(sysm)
    prec = getattr(ib, precision_name)
    phi = phi64 if prec == ib.F64 else phi64.converted(prec)
    ref = ham(phi).matrix()
    host_in = np.ascontiguousarray(phi.matrix())
    host_out = np.zeros_like(host_in)
    ham.apply_host(host_in, host_out)
    err = np.linalg.norm(host_out - ref) / np.linalg.norm(ref)
    assert err < tol, err


def test_apply_host_pinned_buffers_and_repeat(c1):
    import torch
    ib, basis, ham, phi64 = c1
    phi = phi64.converted(ib.F32)
    ref = ham(phi).matrix()
    n, s = ref.shape
    host_in = torch.empty((n, s), dtype=torch.complex64, pin_memory=True).numpy()
    host_out = torch.empty((n, s), dtype=torch.complex64, pin_memory=True).numpy()
    host_in[...] = phi.matrix()
    first = ham.apply_host(host_in, host_out, block_states=16).copy()
    second = ham.apply_host(host_in, host_out, block_states=16)
    assert np.array_equal(first, second)
    assert np.linalg.norm(first - ref) / np.linalg.norm(ref) < 2e-6


def test_apply_host_rejects_bad_arguments(c1):
    from inq_b200._lib import InqbError
    ib, basis, ham, phi64 = c1
    a = np.zeros((basis.size(), 8), np.complex128)
    with pytest.raises(InqbError):
        ham.ctx.check(ham.ctx.lib.inqb_apply_host(ham.handle, 8, None, 5, ib.F64, a.ctypes.data, a.ctypes.data, 0))


@pytest.mark.parametrize("precision_name", ["F64", "F32"])
def test_apply_host_many_matches_single_calls(c1, precision_name):
    """inqb_apply_host_many over three sets (one pipeline of state blocks across the sets) gives bitwise
    the results of one inqb_apply_host call per set; an output that aliases an input is refused."""
    import torch
    from inq_b200._lib import InqbError
    ib, basis, ham, phi64 = c1
    prec = getattr(ib, precision_name)
    phi = phi64 if prec == ib.F64 else phi64.converted(prec)
    m = phi.matrix()
    n, s = m.shape
    dt = torch.complex128 if prec == ib.F64 else torch.complex64
    ins = [torch.empty((n, s), dtype=dt, pin_memory=True).numpy() for _ in range(3)]
    outs = [torch.empty((n, s), dtype=dt, pin_memory=True).numpy() for _ in range(3)]
    for k, a in enumerate(ins):
        a[...] = m * (1.0 + 0.5 * k) + (0.25j * k) * np.roll(m, k, axis=1)
    singles = []
    for a in ins:
        o = np.empty_like(a)
        ham.apply_host(a, o, block_states=16)
        singles.append(o)
    ham.apply_host_many(ins, outs, block_states=16)
    for a, b in zip(singles, outs):
        assert np.array_equal(a, b)
    with pytest.raises(InqbError):
        ham.apply_host_many([ins[0], ins[1]], [outs[0], ins[0]])
