"""GPU tests of the device-side projector setup for moving atoms.

ks_hamiltonian::update_projectors (spherical_grid.hpp:59-160, projector.hpp:38-66, called from
etrs.hpp:45-48 when ions move) built by kernels is compared with the host construction, which the
oracle pins (sphere sizes 257 / 15963 of the reference's spherical_grid test):

* sphere points, float32 offsets and sphere sizes are identical;
* projector values agree to 1e-14 relative (the device exp and the host exp may differ in the
  last bit);
* the per-grid-point hit lists are identical: with the device-built values given back through the
  generic table call (whose hit lists the host builds), H|psi> is bitwise the same;
* moving the atoms rebuilds the same tables as a fresh host build at the new positions.

Cells: cubic, a skewed (non-orthogonal) cell and a small cell whose spheres reach several
periodic images.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(ib, lattice, sizes, natoms, radius, rng):
    cell = ib.Cell(np.asarray(lattice, dtype=np.float64))
    rs = ib.RealSpace(cell, sizes=sizes)
    pos = rng.uniform(-0.6, 0.6, (natoms, 3)) @ np.asarray(lattice, dtype=np.float64)
    kb = rng.uniform(-1, 1, (natoms, 4, 4))
    kb = 0.5 * (kb + kb.transpose(0, 2, 1))
    return rs, pos, kb


CASES = [
    ("cubic", np.eye(3) * 10.26, (32, 32, 32), 8, 2.0),
    ("skewed", [[9.0, 0.0, 0.0], [2.5, 8.5, 0.0], [1.0, 1.5, 9.5]], (30, 28, 32), 6, 2.2),
    ("images", np.eye(3) * 4.0, (20, 20, 20), 3, 3.1),
]


@pytest.mark.parametrize("name,lattice,sizes,natoms,radius", CASES)
def test_device_tables_match_host(rng, name, lattice, sizes, natoms, radius):
    import inq_b200 as ib
    rs, pos, kb = _system(ib, lattice, sizes, natoms, radius, rng)
    hh = ib.KSHamiltonian(rs)
    hh.update_projectors_gaussian(pos, radius, 0.9, kb)
    hd = ib.KSHamiltonian(rs)
    hd.update_projectors_gaussian(pos, radius, 0.9, kb, device=True)
    assert hh.projectors_info() == hd.projectors_info()
    p_h, x_h, m_h, n_h = hh.projector_tables()
    p_d, x_d, m_d, n_d = hd.projector_tables()
    assert np.array_equal(n_h, n_d)
    assert np.array_equal(p_h, p_d)
    assert np.array_equal(x_h.view(np.uint32), x_d.view(np.uint32))
    scale = np.max(np.abs(m_h))
    assert np.max(np.abs(m_h - m_d)) <= 1e-14 * scale

    # hit lists: the device-built values through the generic call (host-built hit lists) give
    # bitwise the same operator as the device-built Hamiltonian
    hg = ib.KSHamiltonian(rs)
    hg.set_projectors(p_d, x_d, m_d, kb, n_d, np.full(natoms, 4, np.int32))
    x = rng.standard_normal(tuple(sizes) + (5,)) + 1j * rng.standard_normal(tuple(sizes) + (5,))
    phi = ib.OrbitalSet.from_array(rs, x)
    a = hd(phi).matrix()
    b = hg(phi).matrix()
    assert np.array_equal(a, b)
    c = hh(phi).matrix()
    assert np.linalg.norm(a - c) <= 1e-13 * np.linalg.norm(c)


def test_moving_atoms_rebuilds_the_tables(rng):
    import inq_b200 as ib
    lattice = np.eye(3) * 10.26
    rs, pos, kb = _system(ib, lattice, (32, 32, 32), 8, 2.0, rng)
    ham = ib.KSHamiltonian(rs)
    ham.update_projectors_gaussian(pos, 2.0, 0.9, kb)
    x = rng.standard_normal((32, 32, 32, 4)) + 1j * rng.standard_normal((32, 32, 32, 4))
    phi = ib.OrbitalSet.from_array(rs, x)
    for step in range(3):
        pos = pos + rng.normal(0.0, 0.15, pos.shape)
        ham.move_atoms(pos)
        ref = ib.KSHamiltonian(rs)
        ref.update_projectors_gaussian(pos, 2.0, 0.9, kb)
        p_m, x_m, _, n_m = ham.projector_tables()
        p_r, x_r, _, n_r = ref.projector_tables()
        assert np.array_equal(n_m, n_r) and np.array_equal(p_m, p_r) and np.array_equal(x_m, x_r)
        a = ham(phi).matrix()
        b = ref(phi).matrix()
        assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(b)


def test_move_needs_a_gaussian_build(rng):
    import inq_b200 as ib
    rs = ib.RealSpace(ib.Cell.cubic(8.0), sizes=(16, 16, 16))
    ham = ib.KSHamiltonian(rs)
    with pytest.raises(Exception):
        ham.move_atoms(np.zeros((0, 3)))
    ham.update_projectors_gaussian(np.zeros((2, 3)), 1.5, 0.8, np.zeros((2, 4, 4)), device=True)
    with pytest.raises(ValueError):
        ham.move_atoms(np.zeros((3, 3)))


def test_device_setup_of_the_96_grid_system():
    """The 64-atom 96^3 system: the device build equals the host build."""
    import inq_b200 as ib
    from inq_b200 import synthetic
    sysm = synthetic.config("c2", nst=4)
    rs = ib.RealSpace(ib.Cell(sysm.lattice), sizes=sysm.sizes)
    hh = ib.KSHamiltonian(rs)
    hh.update_projectors_gaussian(sysm.positions, sysm.radius, sysm.rc, sysm.kb)
    hd = ib.KSHamiltonian(rs)
    hd.update_projectors_gaussian(sysm.positions, sysm.radius, sysm.rc, sysm.kb, device=True)
    p_h, x_h, m_h, n_h = hh.projector_tables()
    p_d, x_d, m_d, n_d = hd.projector_tables()
    assert np.array_equal(n_h, n_d) and np.array_equal(p_h, p_d) and np.array_equal(x_h, x_d)
    assert np.max(np.abs(m_h - m_d)) <= 1e-14 * np.max(np.abs(m_h))
