"""GPU parity at the benchmark constructions, against the FP64 oracle.

The operator does not couple states, so a slice of a configuration's states is an exact check of
the kernels the benchmark runs on it.  The slices keep every pass of H on the kernels the full
configuration uses: 64 states give 1024-byte (FP64) and 512-byte (FP32) rows, so the TMA FFT
passes (96- and 120-point codelets, digit-reversed z order, 512-byte-row streaming passes of the
mixed form) and the bulk-copy nonlocal kernels run.

* 96^3 grid, a = 20.52 bohr, 64 jittered atoms (2x2x2 diamond supercell), 64 states;
* 120^3 grid, a = 25.6 bohr, 128 jittered atoms, 64 states (16 for the ETRS step).

Tolerances: plain FP64 form <= 1e-12 relative in H|psi> (ks_hamiltonian.hpp:137-156); mixed form
<= 1e-6 relative in H|psi> and eigenvalues within 1e-6 Ha (energy.hpp:83-89) of the oracle; one
ETRS step (etrs.hpp:22-79) <= 1e-11 relative in the orbitals and density.
"""

import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL_MIXED = 1e-6
TOL_EIG = 1e-6


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def _oracle(sysm):
    rs = O.RealSpace(O.Cell(sysm.lattice), sysm.sizes)
    pa = O.ProjectorAll.pack([O.build_projector(rs, R, sysm.radius, sysm.rc, sysm.kb[a])
                              for a, R in enumerate(sysm.positions)])
    return O.Hamiltonian(rs, sysm.local_potential(), pa, np.zeros(3)), rs


def _system(name, nst):
    from inq_b200 import synthetic
    O.set_fft_workers(os.cpu_count() or 1)
    sysm = synthetic.config(name, nst=nst)
    basis, ham, phi = synthetic.build(sysm)
    oh, ors = _oracle(sysm)
    x = phi.hypercubic()
    return dict(sysm=sysm, basis=basis, ham=ham, phi=phi, oh=oh, ors=ors, x=x, ref=oh.apply_real(x),
                eig=O.eigenvalues(oh, x)[0])


@pytest.fixture(scope="module")
def c2():
    s = _system("c2", 64)
    yield s
    O.set_fft_workers(None)


@pytest.fixture(scope="module")
def c3():
    s = _system("c3", 64)
    yield s
    O.set_fft_workers(None)


def _check_fp64(ib, s, nl_bulk):
    ctx = s["basis"].ctx
    ctx.set_option("nl_bulk", nl_bulk)
    try:
        h = s["ham"](s["phi"]).hypercubic()
    finally:
        ctx.set_option("nl_bulk", 0)
    assert rel(h, s["ref"]) < TOL64


def _check_mixed(ib, s, nl_bulk):
    ctx = s["basis"].ctx
    ctx.set_option("nl_bulk", nl_bulk)
    try:
        p32 = s["phi"].converted(ib.F32)
        h = s["ham"](p32).hypercubic()
        eig, _ = s["ham"].eigenvalues(p32)
    finally:
        ctx.set_option("nl_bulk", 0)
    # against the oracle on the FP64 orbitals (the rounding of the input to FP32 included) and on the
    # FP32-rounded orbitals the device holds (the arithmetic of the mixed form alone)
    err = rel(h, s["ref"])
    x32 = p32.hypercubic().astype(np.complex128)
    err_arith = rel(h, s["oh"].apply_real(x32))
    deig = float(np.max(np.abs(eig - s["eig"])))
    print(f"mixed H rel err {err:.3e} (arithmetic alone {err_arith:.3e}), eigenvalues {deig:.3e} Ha")
    assert err < TOL_MIXED
    assert err_arith < TOL_MIXED
    assert deig < TOL_EIG


@pytest.mark.parametrize("nl_bulk", [0, 1, -1])
def test_c2_fp64_parity(c2, nl_bulk):
    import inq_b200 as ib
    _check_fp64(ib, c2, nl_bulk)


@pytest.mark.parametrize("nl_bulk,fft_wide", [(0, 1), (1, 1), (0, 0)])
def test_c2_mixed_parity(c2, nl_bulk, fft_wide):
    import inq_b200 as ib
    c2["basis"].ctx.set_option("fft_wide", fft_wide)
    try:
        _check_mixed(ib, c2, nl_bulk)
    finally:
        c2["basis"].ctx.set_option("fft_wide", 1)


def test_c2_fp64_eigenvalues(c2):
    eig, _ = c2["ham"].eigenvalues(c2["phi"])
    assert np.max(np.abs(eig - c2["eig"])) < 1e-10


@pytest.mark.parametrize("nl_bulk", [0, 1])
def test_c3_fp64_parity(c3, nl_bulk):
    import inq_b200 as ib
    _check_fp64(ib, c3, nl_bulk)


def test_c3_mixed_parity(c3):
    import inq_b200 as ib
    _check_mixed(ib, c3, 0)


def test_c3_etrs_step_parity():
    """One ETRS step at 120^3 with 128 atoms (16 states: 256-byte FP64 rows, the TMA passes) against the
    oracle, at the Taylor-stable time step of the grid."""
    import inq_b200 as ib
    from inq_b200 import synthetic
    O.set_fft_workers(os.cpu_count() or 1)
    try:
        sysm = synthetic.config("c3", nst=16)
        basis, ham, phi = synthetic.build(sysm)
        oh, ors = _oracle(sysm)
        x = phi.hypercubic()
        occ = np.full(sysm.nst, 2.0)
        dt = synthetic.taylor_stable_dt(sysm)
        dens, dip, iters = ib.etrs(ham, [phi], [occ], dt, want_density=True)
        ref, rdens, riters = O.etrs_step(oh, [x], [occ], dt)
        assert iters == riters
        assert rel(phi.hypercubic(), ref[0]) < 1e-11
        assert rel(dens.reshape(sysm.sizes), rdens) < 1e-11
        assert np.max(np.abs(dip - O.dipole_electronic(ors, rdens))) < 1e-9
    finally:
        O.set_fft_workers(None)
