"""GPU parity of the Fourier-space eigensolver step against the FP64 oracle.

eigensolvers::steepest_descent (steepest_descent.hpp:23-86) with the Teter-Payne-Allan
preconditioner (preconditioner.hpp:24-46) and the final orthogonalize, on a Fourier-space set as
ground_state/calculator.hpp:161-174 calls it: the updated set to 1e-10 relative, and repeated
steps lower the sum of the eigenvalues."""

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.fixture(scope="module")
def c1():
    import inq_b200 as ib
    from inq_b200 import synthetic
    sysm = synthetic.config("c1", nst=8)
    basis, ham, phi = synthetic.build(sysm)
    cell = O.Cell(sysm.lattice)
    ors = O.RealSpace(cell, sysm.sizes)
    pa = O.ProjectorAll.pack([O.build_projector(ors, R, sysm.radius, sysm.rc, sysm.kb[a])
                              for a, R in enumerate(sysm.positions)])
    oh = O.Hamiltonian(ors, sysm.local_potential(), pa)
    return ib, sysm, basis, ham, phi, oh, ors


def test_steepest_descent_parity(c1):
    ib, sysm, basis, ham, phi, oh, ors = c1
    fphi = ib.to_fourier(phi)
    ref = O.steepest_descent(oh, O.to_fourier(phi.hypercubic()))
    ham.steepest_descent(fphi)
    assert rel(fphi.hypercubic(), ref) < 1e-10
    # orthonormal in the Fourier inner product
    s = ib.overlap(fphi)
    assert np.max(np.abs(s - np.eye(sysm.nst))) < 1e-12


def test_steepest_descent_lowers_the_energy(c1):
    ib, sysm, basis, ham, phi, oh, ors = c1
    p = phi.copy()
    sums = []
    for _ in range(3):
        e, _ = ham.eigenvalues(p)
        sums.append(float(np.sum(e)))
        f = ib.to_fourier(p)
        ham.steepest_descent(f)
        p = ib.to_real(f)
    assert sums[1] < sums[0] and sums[2] < sums[1]
