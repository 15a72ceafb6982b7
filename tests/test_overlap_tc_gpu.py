"""GPU tests of the tensor-core overlap of single-precision orbital sets.

operations::overlap (overlap.hpp:26-95) of FP32 sets runs as split-BF16 products on the
tcgen05 tensor cores with FP32 accumulation and an FP64 sum of the per-SM partials.  The
result is compared with the exact overlap of the same FP32 values formed in float64 on the
host.  The two-term split keeps 16 significant bits of every value, so the error of S_ij is
bounded relative to |a_i| |b_j| (the normwise bound of an inner product), not to |S_ij|, which
for nearly orthogonal states is far smaller: max_ij |dS_ij| / (|a_i| |b_j|) <= 1e-6.  For the
sums that are large (norms, a set with itself) the relative error is checked too.  Shapes cover
one and several 128-state blocks, a state count that is not a multiple of 16, unequal set sizes,
and more than 256 states of b.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _set(ib, rs, rng, nst, precision):
    sizes = rs.sizes
    arr = rng.standard_normal(tuple(sizes) + (nst,)) + 1j * rng.standard_normal(tuple(sizes) + (nst,))
    return ib.OrbitalSet.from_array(rs, arr, precision=precision)


def _exact(rs, a, b):
    """dV a^H b in float64 from the sets' stored (single-precision) values."""
    A = a.matrix().astype(np.complex128)
    B = b.matrix().astype(np.complex128)
    return rs.volume_element() * (A.conj().T @ B)


def _normwise(rs, a, b, got, ref):
    """max_ij |got - ref|_ij / (|a_i| |b_j|), the norms with the volume element."""
    na = np.sqrt(rs.volume_element() * np.sum(np.abs(a.matrix().astype(np.complex128)) ** 2, axis=0))
    nb = np.sqrt(rs.volume_element() * np.sum(np.abs(b.matrix().astype(np.complex128)) ** 2, axis=0))
    return float(np.max(np.abs(got - ref) / np.outer(na, nb)))


@pytest.mark.parametrize("sizes,na,nb", [((20, 18, 16), 64, 64), ((24, 24, 20), 160, 96),
                                         ((16, 16, 12), 40, 300), ((18, 16, 16), 13, 29)])
def test_tensor_core_overlap_matches_fp64(sizes, na, nb, rng):
    import inq_b200 as ib
    rs = ib.RealSpace(ib.Cell.cubic(7.5), sizes=sizes)
    a = _set(ib, rs, rng, na, ib.F32)
    b = _set(ib, rs, rng, nb, ib.F32)
    ref = _exact(rs, a, b)
    got = ib.overlap(a, b)
    assert got.shape == (na, nb)
    err = _normwise(rs, a, b, got, ref)
    assert err < TOL, err
    # a set with itself: the norms on the diagonal to 1e-6 relative
    saa = ib.overlap(a)
    d = np.real(np.diag(saa)) / np.real(np.diag(_exact(rs, a, a))) - 1.0
    assert np.max(np.abs(d)) < TOL
    # the same call again gives bitwise the same matrix (fixed-order partial sums)
    assert np.array_equal(ib.overlap(a, b), got)


def test_tensor_core_and_simt_overlaps_agree(rng):
    import inq_b200 as ib
    rs = ib.RealSpace(ib.Cell.cubic(8.0), sizes=(24, 20, 20))
    a = _set(ib, rs, rng, 96, ib.F32)
    tc = ib.overlap(a)
    rs.ctx.set_option("overlap_tc", 0)
    try:
        simt = ib.overlap(a)
    finally:
        rs.ctx.set_option("overlap_tc", 1)
    assert _normwise(rs, a, a, tc, simt) < TOL
    # Hermitian to the accuracy of the products
    assert _normwise(rs, a, a, tc, tc.conj().T) < TOL


def test_single_precision_orthogonalize_on_tensor_cores(rng):
    """orthogonalize.hpp:25-41 with the tensor-core overlap and the FP64 Cholesky: the stored
    FP32 set is orthonormal to single-precision accuracy."""
    import inq_b200 as ib
    rs = ib.RealSpace(ib.Cell.cubic(9.0), sizes=(24, 24, 24))
    phi = _set(ib, rs, rng, 48, ib.F32)
    ib.orthogonalize(phi)
    s = _exact(rs, phi, phi)
    assert np.max(np.abs(s - np.eye(48))) < 2e-6
