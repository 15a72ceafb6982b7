"""GPU parity of the CUDA path (through the C ABI) against the FP64 CPU oracle.

Tolerances (written here, checked per test):
  * plain FP64 form: relative Frobenius error <= 1e-12 in H|psi>, FFTs and every
    derived array; energies within 1e-10 Ha;
  * mixed form (FP32 orbitals): relative error <= 2e-6 against the FP64 oracle.
"""

import math

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-6


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.fixture(scope="module")
def ib():
    import inq_b200
    return inq_b200


def _random_orbitals(rng, sizes, nst):
    return (rng.standard_normal(tuple(sizes) + (nst,)) + 1j * rng.standard_normal(tuple(sizes) + (nst,)))


# ------------------------------------------------------------------ transforms

@pytest.mark.parametrize("impl", [0, 1])
@pytest.mark.parametrize("sizes,nst", [((20, 20, 20), 6), ((32, 32, 32), 16), ((18, 24, 20), 13), ((54, 54, 54), 7),
                                       ((14, 21, 28), 3), ((24, 40, 30), 33), ((96, 96, 96), 18), ((120, 8, 10), 40),
                                       ((64, 72, 48), 32), ((128, 24, 40), 17)])
def test_fft_roundtrip_and_parity(ib, rng, sizes, nst, impl):
    """to_fourier / to_real (transform.hpp:52-249) vs numpy's FFT; radices 2,3,4,5,7,8; both FFT kernels."""
    cell = ib.Cell.orthorhombic(9.0, 12.0, 10.0)
    rs = ib.RealSpace(cell, sizes=sizes)
    rs.ctx.set_option("fft_impl", impl)
    try:
        x = _random_orbitals(rng, sizes, nst)
        phi = ib.OrbitalSet.from_array(rs, x)
        f = ib.to_fourier(phi)
        assert rel(f.hypercubic(), O.to_fourier(x)) < TOL64
        back = ib.to_real(f)
        assert rel(back.hypercubic(), x) < TOL64
        un = ib.to_real(f, normalize=False)
        assert rel(un.hypercubic(), x * np.prod(sizes)) < TOL64
        rs.ctx.synchronize()
    finally:
        rs.ctx.set_option("fft_impl", 0)


@pytest.mark.parametrize("mixed_compute", [1, 0])
@pytest.mark.parametrize("impl", [0, 1])
@pytest.mark.parametrize("sizes,nst", [((48, 40, 36), 64), ((96, 96, 96), 32), ((24, 32, 72), 40),
                                       ((96, 96, 96), 64), ((40, 48, 120), 72), ((96, 96, 96), 33),
                                       ((72, 64, 48), 65), ((24, 120, 40), 127)])
def test_fft_mixed_precision_kernels(ib, rng, sizes, nst, impl, mixed_compute):
    """FP32 transforms through both kernels: relative error <= 2e-6 against the FP64 oracle (64 and 72
    states: the 512-byte-row streaming passes, the second tile of 72 states partly outside the set; an
    odd number of states: rows that are not 16-byte multiples, copied by the producer warp)."""
    rs = ib.RealSpace(ib.Cell.cubic(10.0), sizes=sizes)
    rs.ctx.set_option("fft_impl", impl)
    rs.ctx.set_option("mixed_compute", mixed_compute)
    try:
        x = _random_orbitals(rng, sizes, nst)
        phi = ib.OrbitalSet.from_array(rs, x, precision=ib.F32)
        f = ib.to_fourier(phi)
        assert rel(f.hypercubic(), O.to_fourier(x)) < TOL32
        assert rel(ib.to_real(f).hypercubic(), x) < TOL32
    finally:
        rs.ctx.set_option("fft_impl", 0)
        rs.ctx.set_option("mixed_compute", 0)


def test_fft_mixed_precision(ib, rng):
    sizes, nst = (48, 40, 36), 20
    rs = ib.RealSpace(ib.Cell.cubic(10.0), sizes=sizes)
    x = _random_orbitals(rng, sizes, nst)
    phi = ib.OrbitalSet.from_array(rs, x, precision=ib.F32)
    f = ib.to_fourier(phi)
    assert rel(f.hypercubic(), O.to_fourier(x)) < TOL32


def test_laplacian_plane_wave(ib):
    """laplacian.hpp:143-200 on the device: (s+1) e^{ik.r} -> factor (-k^2) (s+1) e^{ik.r}."""
    cell = ib.Cell.orthorhombic(9.0, 12.0, 10.0)
    rs = ib.RealSpace(cell, spacing=0.49672941)
    r = rs.rvector_cartesian()
    kvec = 2.0 * math.pi * np.array([1.0 / 9, 1.0 / 12, 1.0 / 10])
    ff = np.exp(1j * (r @ kvec))
    s1 = np.arange(13) + 1.0
    func = s1 * ff[..., None]
    factor = 0.673214
    lap = ib.to_real(ib.laplacian(ib.to_fourier(ib.OrbitalSet.from_array(rs, func)), factor)).hypercubic()
    an = s1 * factor * (-kvec @ kvec) * ff[..., None]
    assert np.sum(np.abs(lap - an)) < 1e-8


# ------------------------------------------------------------------ reference known answers through the GPU

def _pw10(ib):
    return ib.RealSpace(ib.Cell.cubic(10.0), spacing=0.49672941)


def test_known_answers_free_and_oscillator(ib):
    """ks_hamiltonian.hpp:324-536: constant -> 0, plane waves -> k^2/2, oscillator 0.0051420503."""
    rs = _pw10(ib)
    assert rs.sizes == (20, 20, 20)
    nst = 6
    ham = ib.KSHamiltonian(rs)
    ham.set_scalar_potential(np.zeros(rs.sizes))
    h = ham(ib.OrbitalSet.from_array(rs, np.ones(rs.sizes + (nst,), complex))).hypercubic()
    assert np.sum(np.abs(h)) / h.size < 1e-14
    kk = 2.0 * math.pi / 10.0
    x = rs.rvector_cartesian()[..., 0]
    s = np.arange(nst)
    pw = np.exp(1j * s * kk * x[..., None])
    h = ham(ib.OrbitalSet.from_array(rs, pw)).hypercubic()
    assert np.sum(np.abs(h - 0.5 * (s * kk) ** 2 * pw)) / h.size < 1e-14
    # Fourier-space operator
    hf = ib.to_real(ham(ib.to_fourier(ib.OrbitalSet.from_array(rs, pw)))).hypercubic()
    assert np.sum(np.abs(hf - 0.5 * (s * kk) ** 2 * pw)) / hf.size < 1e-14
    ww = 2.0
    r = rs.rvector_cartesian()
    r2 = np.sum(r * r, axis=-1)
    ham.set_scalar_potential(0.5 * ww * ww * r2)
    phi = np.repeat(np.exp(-ww * r2)[..., None], nst, axis=-1).astype(complex)
    h = ham(ib.OrbitalSet.from_array(rs, phi)).hypercubic()
    diff = np.sum(np.abs(h - 1.5 * ww * phi)) / h.size
    assert abs(diff - 0.0051420503) < 1.2e-5 * 0.0051420503
    hf = ib.to_real(ham(ib.to_fourier(ib.OrbitalSet.from_array(rs, phi)))).hypercubic()
    diff = np.sum(np.abs(hf - 1.5 * ww * phi)) / hf.size
    assert abs(diff - 0.0051420503) < 1.2e-5 * 0.0051420503


# ------------------------------------------------------------------ full operator on a synthetic system

def _oracle_system(sysm, A=(0.0, 0.0, 0.0)):
    cell = O.Cell(sysm.lattice)
    rs = O.RealSpace(cell, sysm.sizes)
    projs = []
    for a, R in enumerate(sysm.positions):
        projs.append(O.build_projector(rs, R, sysm.radius, sysm.rc, sysm.kb[a]))
    pa = O.ProjectorAll.pack(projs)
    V = sysm.local_potential()
    return O.Hamiltonian(rs, V, pa, np.asarray(A, float)), rs


@pytest.fixture(scope="module")
def c1(ib):
    from inq_b200 import synthetic
    sysm = synthetic.config("c1")
    basis, ham, phi = synthetic.build(sysm)
    oh, ors = _oracle_system(sysm)
    return sysm, basis, ham, phi, oh, ors


def test_projector_tables_match_oracle(c1):
    sysm, basis, ham, phi, oh, ors = c1
    points, pos, mats, npts = ham.projector_tables()
    pa = oh.pa
    assert np.array_equal(npts, pa.npts)
    assert np.array_equal(points, pa.points)
    assert np.array_equal(pos, pa.positions)
    assert rel(mats, pa.matrices) < 1e-15


def test_orbitals_orthonormal(ib, c1):
    sysm, basis, ham, phi, oh, ors = c1
    S = ib.overlap(phi)
    assert np.max(np.abs(S - np.eye(sysm.nst))) < 1e-12
    x = phi.hypercubic()
    assert np.max(np.abs(O.overlap(ors, x) - np.eye(sysm.nst))) < 1e-12


@pytest.mark.parametrize("kpoint,A", [((0.0, 0.0, 0.0), (0.0, 0.0, 0.0)), ((0.3, -0.2, 0.1), (0.0, 0.0, 0.0)),
                                      ((0.0, 0.0, 0.0), (0.05, 0.0, -0.02))])
def test_hamiltonian_real_parity(ib, c1, kpoint, A):
    """ks_hamiltonian::operator()(real space) vs the oracle: rel err <= 1e-12 (C1: 32^3, 16 states, 8 atoms)."""
    sysm, basis, ham, phi, oh, ors = c1
    x = phi.hypercubic()
    ph = ib.OrbitalSet.from_array(basis, x, kpoint=kpoint)
    ham.uniform_vector_potential = np.asarray(A)
    try:
        h = ham(ph).hypercubic()
    finally:
        ham.uniform_vector_potential = np.zeros(3)
    oh.A_cov = np.asarray(A, float)
    ref = oh.apply_real(x, kpoint)
    oh.A_cov = np.zeros(3)
    assert rel(h, ref) < TOL64


def test_hamiltonian_fourier_parity(ib, c1):
    sysm, basis, ham, phi, oh, ors = c1
    x = phi.hypercubic()
    kp = (0.1, 0.2, -0.3)
    fx = O.to_fourier(x)
    fph = ib.OrbitalSet.from_array(basis, fx, kpoint=kp, space=ib.FOURIER_SPACE)
    h = ham(fph).hypercubic()
    assert rel(h, oh.apply_fourier(fx, kp)) < TOL64


@pytest.fixture(scope="module")
def c1big(ib):
    """C1 construction with 64 states: every FFT axis and state count goes through the TMA kernels."""
    from inq_b200 import synthetic
    sysm = synthetic.config("c1", nst=64)
    basis, ham, phi = synthetic.build(sysm)
    oh, ors = _oracle_system(sysm)
    return sysm, basis, ham, phi, oh, ors


@pytest.mark.parametrize("impl", [0, 1])
def test_hamiltonian_kernels_both_paths(ib, c1big, impl):
    """Real- and Fourier-form H through the specialised (0) and generic (1) FFT kernels, FP64 and FP32."""
    sysm, basis, ham, phi, oh, ors = c1big
    basis.ctx.set_option("fft_impl", impl)
    try:
        x = phi.hypercubic()
        kp = (0.2, -0.1, 0.05)
        ref = oh.apply_real(x, kp)
        h = ham(ib.OrbitalSet.from_array(basis, x, kpoint=kp)).hypercubic()
        assert rel(h, ref) < TOL64
        h32 = ham(ib.OrbitalSet.from_array(basis, x, kpoint=kp, precision=ib.F32)).hypercubic()
        assert rel(h32, ref) < TOL32
        fx = O.to_fourier(x)
        hf = ham(ib.OrbitalSet.from_array(basis, fx, kpoint=kp, space=ib.FOURIER_SPACE)).hypercubic()
        assert rel(hf, oh.apply_fourier(fx, kp)) < TOL64
        p = phi.copy()
        ib.exponential_in_place(ham, complex(0.0, -0.025), p)
        assert rel(p.hypercubic(), O.exponential_in_place(oh.apply_real, complex(0.0, -0.025), x)) < TOL64
        basis.ctx.synchronize()
    finally:
        basis.ctx.set_option("fft_impl", 0)


@pytest.mark.parametrize("nst", [33, 65, 97])
def test_hamiltonian_odd_state_count_single(ib, nst):
    """Mixed-form H|psi> of an odd number of states (rows of 8 mod 16 bytes, which TMA cannot move: the
    producer warp copies them with 8-byte cp.async) against the oracle, 2e-6 relative, with k and A, and
    within 1e-6 of the same states inside an even-sized set (whose 16-byte rows take the bulk-copy
    nonlocal apply, which fuses its complex multiply-adds)."""
    from inq_b200 import synthetic
    sysm = synthetic.config("c1", nst=nst + 1)
    basis, ham, phi = synthetic.build(sysm)
    oh, ors = _oracle_system(sysm, A=(0.03, 0.0, -0.01))
    ham.uniform_vector_potential = np.array([0.03, 0.0, -0.01])
    try:
        x = phi.hypercubic()[..., :nst]
        kp = (0.1, -0.2, 0.05)
        h = ham(ib.OrbitalSet.from_array(basis, x, kpoint=kp, precision=ib.F32)).hypercubic()
        assert rel(h, oh.apply_real(x, kp)) < TOL32
        h_even = ham(ib.OrbitalSet.from_array(basis, phi.hypercubic(), kpoint=kp, precision=ib.F32)).hypercubic()
        assert rel(h, h_even[..., :nst]) < 1e-6
        # a real-time step runs through the same passes (Horner steps and the kept Taylor terms)
        p = ib.OrbitalSet.from_array(basis, x, kpoint=kp, precision=ib.F32)
        occ = np.full(nst, 2.0)
        dens, dip, iters = ib.etrs(ham, [p], [occ], 0.01, want_density=True)
        ref, rdens, riters = O.etrs_step(oh, [x], [occ], 0.01, kpoints=[kp])
        assert rel(p.hypercubic(), ref[0]) < 1e-5
    finally:
        ham.uniform_vector_potential = np.zeros(3)


@pytest.mark.parametrize("precision,mixed_compute,nst", [("F32", 0, 33), ("F32", 0, 40), ("F32", 0, 64),
                                                          ("F32", 0, 100), ("F32", 1, 33), ("F32", 1, 72),
                                                          ("F64", 0, 17), ("F64", 0, 40)])
def test_flat_columns_match_line_tiles(ib, rng, precision, mixed_compute, nst):
    """The y and x passes over flattened (point, state) columns (option fft_flat, the default) against
    tiles of one line times a block of states: H|psi> (kinetic factors of two lines inside one tile
    included) and to_fourier / to_real agree to rounding, and with the oracle, for odd, ragged and
    whole-tile state counts."""
    from inq_b200 import synthetic
    sysm = synthetic.config("c1", nst=nst)
    prec = getattr(ib, precision)
    basis, ham, phi = synthetic.build(sysm, precision=prec)
    ctx = basis.ctx
    oh, ors = _oracle_system(sysm)
    tol = TOL32 if prec == ib.F32 else TOL64
    ctx.set_option("mixed_compute", mixed_compute)
    try:
        x = phi.hypercubic().astype(np.complex128)
        h_flat = ham(phi).hypercubic()
        f_flat = ib.to_fourier(phi).hypercubic()
        ctx.set_option("fft_flat", 0)
        h_line = ham(phi).hypercubic()
        f_line = ib.to_fourier(phi).hypercubic()
        ctx.set_option("fft_flat", 1)
        assert rel(h_flat, h_line) < (1e-6 if prec == ib.F32 else 1e-14)
        assert rel(f_flat, f_line) < (1e-6 if prec == ib.F32 else 1e-14)
        assert rel(h_flat, oh.apply_real(x)) < tol
        assert rel(f_flat, O.to_fourier(x)) < tol
    finally:
        ctx.set_option("fft_flat", 1)
        ctx.set_option("mixed_compute", 0)


def test_hamiltonian_deterministic(ib, c1):
    sysm, basis, ham, phi, oh, ors = c1
    a = ham(phi).matrix()
    b = ham(phi).matrix()
    assert np.array_equal(a, b)


def test_nonlocal_pieces(ib, c1):
    sysm, basis, ham, phi, oh, ors = c1
    x = phi.hypercubic()
    occ = np.full(sysm.nst, 2.0)
    assert rel(ham.non_local(phi).hypercubic(), oh.non_local(x)) < TOL64
    e = ham.non_local_energy(phi, occ)
    assert abs(e - oh.non_local_energy(x, occ)) < 1e-10
    kin = ham.kinetic_expectation_value(phi)
    assert np.max(np.abs(kin - oh.kinetic_expectation_value(x))) < 1e-10
    eig, res = ham.eigenvalues(phi)
    oeig, ores = O.eigenvalues(oh, x)
    assert np.max(np.abs(eig - oeig)) < 1e-10
    assert np.max(np.abs(res - ores)) < 1e-9


@pytest.mark.parametrize("mixed_compute", [1, 0])
def test_hamiltonian_mixed_precision(ib, c1big, mixed_compute):
    """Mixed form (FP32 orbitals; FP64 or compensated FP32 butterflies): H|psi> within 2e-6 relative and
    eigenvalues within 1e-6 Ha of the FP64 oracle in both."""
    sysm, basis, ham, phi, oh, ors = c1big
    basis.ctx.set_option("mixed_compute", mixed_compute)
    try:
        x = phi.hypercubic()
        ph32 = phi.converted(ib.F32)
        h = ham(ph32).hypercubic()
        ref = oh.apply_real(x)
        assert rel(h, ref) < TOL32
        eig, _ = ham.eigenvalues(ph32)
        oeig, _ = O.eigenvalues(oh, x)
        assert np.max(np.abs(eig - oeig)) < 1e-6
        if mixed_compute == 1:
            assert rel(h, ref) < 5e-7
    finally:
        basis.ctx.set_option("mixed_compute", 0)


# ------------------------------------------------------------------ real time

def test_exponential_parity(ib, c1):
    sysm, basis, ham, phi, oh, ors = c1
    x = phi.hypercubic()
    p = phi.copy()
    ib.exponential_in_place(ham, complex(0.0, -0.025), p)
    assert rel(p.hypercubic(), O.exponential_in_place(oh.apply_real, complex(0.0, -0.025), x)) < TOL64
    p = phi.copy()
    e1 = ib.exponential_2_for_1(ham, complex(0.0, -0.025), complex(0.0, -0.05), p)
    r1, r2 = O.exponential_2_for_1(oh.apply_real, complex(0.0, -0.025), complex(0.0, -0.05), x)
    assert rel(e1.hypercubic(), r1) < TOL64
    assert rel(p.hypercubic(), r2) < TOL64


def test_density_dipole_kick(ib, c1):
    sysm, basis, ham, phi, oh, ors = c1
    x = phi.hypercubic()
    occ = np.full(sysm.nst, 2.0)
    d = ib.density([phi], [occ]).reshape(sysm.sizes)
    od = O.density([x], [occ])
    assert rel(d, od) < TOL64
    assert np.max(np.abs(ib.dipole(basis, d) - O.dipole_electronic(ors, od))) < 1e-10
    k = phi.copy()
    ib.apply_phase_kick(k, [0.01, 0.0, 0.0])
    assert rel(k.hypercubic(), O.kick_phase(ors, x, [0.01, 0.0, 0.0])) < TOL64


def test_etrs_step_parity(ib, c1):
    """One ETRS step (etrs.hpp:22-79) for the fixed Hamiltonian vs the oracle."""
    sysm, basis, ham, phi, oh, ors = c1
    x = phi.hypercubic()
    occ = np.full(sysm.nst, 2.0)
    p = phi.copy()
    dens, dip, iters = ib.etrs(ham, [p], [occ], 0.05, want_density=True)
    ref, rdens, riters = O.etrs_step(oh, [x], [occ], 0.05)
    assert iters == riters
    assert rel(p.hypercubic(), ref[0]) < TOL64
    assert rel(dens.reshape(sysm.sizes), rdens) < TOL64
    assert np.max(np.abs(dip - O.dipole_electronic(ors, rdens))) < 1e-10
    # the step's dipole is summed on the device; the host form of the same density agrees to rounding
    assert np.max(np.abs(dip - ib.dipole(basis, dens))) < 1e-12 * max(1.0, float(np.max(np.abs(dip))))


def test_subspace_diagonalization(ib, c1):
    """subspace_diagonalization.hpp:21-29 vs the oracle: eigenvalues within 1e-10 Ha, rotated set diagonalises H."""
    sysm, basis, ham, phi, oh, ors = c1
    x = phi.hypercubic()
    p = phi.copy()
    w = ham.subspace_diagonalization(p)
    ow, ox = O.subspace_diagonalization(oh, x)
    assert np.max(np.abs(w - ow)) < 1e-10
    y = p.hypercubic()
    Hs = O.overlap(ors, y, oh.apply_real(y))
    assert np.max(np.abs(Hs - np.diag(ow))) < 1e-9
    assert np.max(np.abs(O.overlap(ors, y) - np.eye(sysm.nst))) < 1e-11


def test_orthogonalize_random(ib, rng):
    rs = ib.RealSpace(ib.Cell.cubic(6.3), spacing=0.44428829)
    x = _random_orbitals(rng, rs.sizes, 40)
    p = ib.OrbitalSet.from_array(rs, x)
    ib.orthogonalize(p)
    S = ib.overlap(p)
    assert np.max(np.abs(S - np.eye(40))) < 1e-13
    ors = O.RealSpace(O.Cell.cubic(6.3), rs.sizes)
    assert rel(p.hypercubic(), O.orthogonalize(ors, x)) < 1e-11
