"""The zero-copy boundary (inqb_orbitals_wrap): orbital sets over caller-owned device memory.

A reference caller's orbital_set already lives on the device (gpu::array,
external_libs/gpurun/include/gpu/array.hpp:66-110), so its ks_hamiltonian::operator()
(ks_hamiltonian.hpp:137-156) must run on that storage without an upload or a download.  Here the
caller's storage is torch's CUDA memory: H through wrapped buffers must equal H through owned sets
bit for bit, in both forms, with no copy of the set made by the library.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    from inq_b200 import synthetic
    sysm = synthetic.config("c1", nst=64)
    basis, ham, phi = synthetic.build(sysm)
    return sysm, basis, ham, phi


@pytest.mark.parametrize("precision_name", ["F64", "F32"])
@pytest.mark.parametrize("space", ["real", "fourier"])
def test_wrapped_apply_is_bitwise_the_owned_apply(c1, precision_name, space):
    import torch

    import inq_b200 as ib
    sysm, basis, ham, phi = c1
    prec = getattr(ib, precision_name)
    src = phi.converted(prec)
    if space == "fourier":
        src = ib.to_fourier(src)
    kp = (0.1, -0.2, 0.05)
    owned_in = ib.OrbitalSet.from_array(basis, src.hypercubic(), kpoint=kp, precision=prec,
                                        space=ib.FOURIER_SPACE if space == "fourier" else ib.REAL_SPACE)
    owned_out = owned_in.skeleton()
    ham.apply(owned_in, owned_out)
    basis.ctx.synchronize()
    expect = owned_out.matrix()
    # device allocations of one owned apply (per-call scratch of the operator from the stream-ordered pool)
    allocs0 = ib.device_alloc_count()
    ham.apply(owned_in, owned_out)
    basis.ctx.synchronize()
    owned_allocs = ib.device_alloc_count() - allocs0

    dtype = torch.complex128 if prec == ib.F64 else torch.complex64
    t_in = torch.from_numpy(src.matrix()).to("cuda")
    t_out = torch.zeros(basis.size(), src.nst, dtype=dtype, device="cuda")
    assert t_in.dtype == dtype
    torch.cuda.synchronize()
    sp = ib.FOURIER_SPACE if space == "fourier" else ib.REAL_SPACE
    w_in = ib.OrbitalSet.from_tensor(basis, t_in, kpoint=kp, space=sp)
    w_out = ib.OrbitalSet.from_tensor(basis, t_out, kpoint=kp, space=sp)
    assert w_in.device_ptr() == t_in.data_ptr() and w_out.device_ptr() == t_out.data_ptr()
    allocs0 = ib.device_alloc_count()
    ham.apply(w_in, w_out)
    basis.ctx.synchronize()
    # wrapping adds no allocation to the operator's own per-call scratch: in particular no copy of either set
    assert ib.device_alloc_count() - allocs0 == owned_allocs
    got = t_out.cpu().numpy()
    assert np.array_equal(got, expect)
    # destroying the wrapped sets leaves the caller's storage alone
    del w_in, w_out
    basis.ctx.synchronize()
    assert np.array_equal(t_out.cpu().numpy(), expect)


def test_wrap_refuses_memory_the_kernels_cannot_use(c1):
    import torch

    import inq_b200 as ib
    from inq_b200._lib import InqbError
    sysm, basis, ham, phi = c1
    n = basis.size() * 4
    host = np.zeros(n, np.complex128)
    with pytest.raises(InqbError, match="device or managed memory"):
        ib.OrbitalSet.wrap(basis, host.ctypes.data, 4)
    pinned = torch.zeros(n, dtype=torch.complex128).pin_memory()
    with pytest.raises(InqbError, match="device or managed memory"):
        ib.OrbitalSet.wrap(basis, pinned.data_ptr(), 4)
    dev = torch.zeros(n + 1, dtype=torch.complex64, device="cuda")
    with pytest.raises(InqbError, match="aligned to 16 bytes"):
        ib.OrbitalSet.wrap(basis, dev.data_ptr() + 8, 4, precision=ib.F32)
    with pytest.raises(ValueError):
        ib.OrbitalSet.from_tensor(basis, torch.zeros(n, dtype=torch.float64, device="cuda"))
