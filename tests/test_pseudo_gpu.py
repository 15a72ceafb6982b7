"""GPU test of H|psi> with projectors built from a UPF pseudopotential.

The device runs the grouped tables of ``pseudo.projector_tables`` (at most four functions per
projector); the oracle runs every atom as one projector with all its functions and the full KB
matrix, as projector.hpp:38-101 builds it.  Two atoms of a synthetic pseudopotential with two
radial projectors for each of l = 0, 1, 2 (18 functions per atom, 5 groups), at a k-point and with a
vector potential: H|psi> agrees to 1e-12 relative (FP64), the nonlocal energy to 1e-10 Ha.
"""

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _synthetic():
    from inq_b200 import pseudo
    r = np.linspace(0.0, 6.0, 601)
    rab = np.full_like(r, r[1] - r[0])
    beta_l, beta, cut = [], [], []
    rng = np.random.default_rng(11)
    for l in range(3):
        for k in range(2):
            rc = 1.3 + 0.2 * l + 0.1 * k
            b = r ** l * np.exp(-(r / (0.5 * rc)) ** 2) * (1.0 + 0.3 * k * r)
            b[r > rc] = 0.0
            beta_l.append(l)
            beta.append(b)
            cut.append(int(np.searchsorted(r, rc)) + 1)
    nb = len(beta_l)
    d = np.zeros((nb, nb))
    for i in range(nb):
        for j in range(i, nb):
            if beta_l[i] == beta_l[j]:
                d[i, j] = d[j, i] = rng.uniform(-2, 2)
    vloc = -2.0 * np.exp(-r ** 2)
    return pseudo.Pseudopotential("Xx", 4.0, r, rab, vloc, beta_l, beta, cut, d)


def test_hamiltonian_with_upf_projectors_matches_oracle(rng):
    import inq_b200 as ib
    from inq_b200 import pseudo
    ps = _synthetic()
    lat = np.diag([8.0, 7.5, 8.5])
    sizes = (24, 20, 24)
    cell = ib.Cell(lat)
    rs = ib.RealSpace(cell, sizes=sizes)
    atoms = [(ps, np.array([1.0, 2.0, -1.5])), (ps, np.array([-3.0, 0.5, 2.5]))]
    points, pos, mats, coeff, npts, nlm, owner = pseudo.projector_tables(cell, sizes, atoms)
    assert len(points) == 10
    ham = ib.KSHamiltonian(rs)
    V = 0.3 * np.cos(2 * np.pi * np.arange(np.prod(sizes)) / 97.0).reshape(sizes)
    ham.set_scalar_potential(V)
    ham.set_projectors(points, pos, mats, coeff, npts, nlm)
    A = np.array([0.01, -0.02, 0.015])
    ham.uniform_vector_potential = A
    kp = (0.1, -0.05, 0.2)
    nst = 6
    x = rng.standard_normal(tuple(sizes) + (nst,)) + 1j * rng.standard_normal(tuple(sizes) + (nst,))
    h = ham(ib.OrbitalSet.from_array(rs, x, kpoint=kp)).hypercubic()

    # oracle: one projector per atom with all 18 functions and the full KB matrix
    ors = O.RealSpace(O.Cell(lat), sizes)
    projs = []
    for p_, R in atoms:
        sph = O.spherical_grid(ors, R, p_.projector_radius())
        cart = ors.cell.contra_to_cart(sph.relpos.astype(np.float64))
        rows = []
        for i, l in enumerate(p_.beta_l):
            rad = pseudo._radial(p_, i, sph.distance.astype(np.float64))
            for y in pseudo.real_ylm(l, cart):
                rows.append(rad * y)
        projs.append(O.Projector(sph, np.array(rows), p_.kb_coefficients()))
    pa = O.ProjectorAll.pack(projs)
    assert pa.matrices.shape[1] == 18
    oh = O.Hamiltonian(ors, V, pa, A)
    ref = oh.apply_real(x, kp)
    err = np.linalg.norm(h - ref) / np.linalg.norm(ref)
    assert err < 1e-12, err
    occ = np.linspace(2.0, 0.5, nst)
    e = ham.non_local_energy(ib.OrbitalSet.from_array(rs, x, kpoint=kp), occ)
    e_ref = oh.non_local_energy(x, occ, kp)
    assert abs(e - e_ref) < 1e-10 * max(1.0, abs(e_ref)), (e, e_ref)


def test_device_built_pseudopotential_projectors(rng):
    """The device kernels build the same projectors as ``projector_tables`` on the host: equal sphere
    points, offsets and sizes, values to 1e-13 relative (the harmonics' last bits), and an H|psi>
    within 1e-13; ``move_atoms`` rebuilds them for new positions like a fresh host build.  Two species
    (18 and 4 functions), a skewed cell."""
    import inq_b200 as ib
    from inq_b200 import pseudo
    ps = _synthetic()
    small = pseudo.Pseudopotential("Yy", 1.0, ps.r, ps.rab, ps.vlocal, [0, 1], [ps.beta[0], ps.beta[2]],
                                   [ps.beta_cutoff[0], ps.beta_cutoff[2]], np.diag([1.5, -0.7]))
    lat = np.array([[8.0, 0.0, 0.0], [1.5, 7.5, 0.0], [0.5, 1.0, 8.5]])
    sizes = (24, 20, 24)
    cell = ib.Cell(lat)
    rs = ib.RealSpace(cell, sizes=sizes)
    atoms = [(ps, np.array([1.0, 2.0, -1.5])), (small, np.array([-3.0, 0.5, 2.5])), (ps, np.array([3.5, -2.0, 1.0]))]
    hh = ib.KSHamiltonian(rs)
    pseudo.set_ions(hh, atoms)
    hd = ib.KSHamiltonian(rs)
    pseudo.set_ions(hd, atoms, device=True)
    assert hh.projectors_info() == hd.projectors_info()
    p_h, x_h, m_h, n_h = hh.projector_tables()
    p_d, x_d, m_d, n_d = hd.projector_tables()
    assert np.array_equal(n_h, n_d) and np.array_equal(p_h, p_d) and np.array_equal(x_h, x_d)
    assert np.max(np.abs(m_h - m_d)) <= 1e-13 * np.max(np.abs(m_h))
    x = rng.standard_normal(tuple(sizes) + (4,)) + 1j * rng.standard_normal(tuple(sizes) + (4,))
    phi = ib.OrbitalSet.from_array(rs, x, kpoint=(0.05, 0.0, -0.1))
    a, b = hd(phi).matrix(), hh(phi).matrix()
    assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(b)
    # moving the atoms
    moved = [(p_, R + rng.normal(0.0, 0.2, 3)) for p_, R in atoms]
    hd.move_atoms(np.array([R for _, R in moved]))
    hr = ib.KSHamiltonian(rs)
    pseudo.set_ions(hr, moved)
    p_m, x_m, m_m, n_m = hd.projector_tables()
    p_r, x_r, m_r, n_r = hr.projector_tables()
    assert np.array_equal(n_m, n_r) and np.array_equal(p_m, p_r) and np.array_equal(x_m, x_r)
    assert np.max(np.abs(m_m - m_r)) <= 1e-13 * np.max(np.abs(m_r))
