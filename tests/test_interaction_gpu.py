"""GPU parity of the interacting Hamiltonian update against the FP64 oracle.

self_consistency::update_hamiltonian (self_consistency.hpp:88-170): V = V_ion + V_H[n] + V_xc[n]
with the periodic Poisson solver (poisson.hpp:98-104) and the LDA (Slater exchange, PZ81
correlation), built on the device from a density.  Checked through the operator it produces
(H|psi> to 1e-12 relative) and the energies (1e-10 Ha), then inside ETRS steps whose
self-consistency loop now rebuilds the potential from every density (etrs.hpp:51, :75)."""

import copy

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


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


@pytest.mark.parametrize("hartree,xc", [(True, "lda"), (True, None), (False, "lda")])
def test_update_hamiltonian_parity(c1, hartree, xc):
    ib, sysm, basis, ham, phi, oh, ors = c1
    occ = np.full(sysm.nst, 2.0)
    vion = sysm.local_potential()
    dens = ib.density([phi], [occ]).reshape(sysm.sizes)
    ham.set_interaction(vion, hartree=hartree, xc=xc)
    try:
        e = ham.update_hamiltonian(dens)
        oh2 = copy.copy(oh)
        oe = O.update_hamiltonian(oh2, vion, dens, hartree=hartree, xc=xc is not None)
        for k in ("external", "hartree", "xc", "nvxc"):
            assert abs(e[k] - oe[k]) < 1e-10, (k, e[k], oe[k])
        assert rel(ham(phi).hypercubic(), oh2.apply_real(phi.hypercubic())) < TOL64
    finally:
        ham.clear_interaction()
        ham.set_scalar_potential(vion)


def test_interacting_etrs_parity(c1):
    """Two ETRS steps with the Hartree + LDA update against the oracle's etrs_step with the same hook."""
    ib, sysm, basis, ham, phi, oh, ors = c1
    from inq_b200 import synthetic
    occ = np.full(sysm.nst, 2.0)
    vion = sysm.local_potential()
    dt = 0.5 * synthetic.taylor_stable_dt(sysm)
    p = phi.copy()
    ib.apply_phase_kick(p, [0.01, 0.0, 0.0])
    x = p.hypercubic()
    ham.set_interaction(vion)
    oh2 = copy.copy(oh)
    try:
        dens0 = ib.density([p], [occ]).reshape(sysm.sizes)
        ham.update_hamiltonian(dens0)
        O.update_hamiltonian(oh2, vion, O.density([x], [occ]))
        hook = lambda n: O.update_hamiltonian(oh2, vion, n)
        for _ in range(2):
            dens, dip, iters = ib.etrs(ham, [p], [occ], dt, want_density=True)
            ref, rdens, riters = O.etrs_step(oh2, [x], [occ], dt, update_hamiltonian=hook)
            x = ref[0]
            assert iters == riters
            assert rel(p.hypercubic(), x) < 1e-11
            assert rel(dens.reshape(sysm.sizes), rdens) < 1e-11
    finally:
        ham.clear_interaction()
        ham.set_scalar_potential(vion)
