"""GPU tests of the bulk-copy forms of the nonlocal kernels (option ``nl_bulk``).

The projection and the apply move whole rows of states through shared memory with bulk
asynchronous copies (``nl_bulk`` 0 chooses them by size, 1 wherever a row is a multiple of 16
bytes, -1 never).  Forced on against forced off, on small systems:

* H|psi> agrees to 1e-14 relative in FP64 (the projection sums the sphere points in another
  grouping) and 2e-6 in single precision;
* with overlapping projectors (five per atom around one centre, so every sphere point has five
  hits) H|psi> also matches the oracle to 1e-12;
* the Taylor exponential, whose apply also updates two accumulators, agrees to 1e-13;
* a single-precision set with an odd state count (rows of 8-byte multiples) takes the register
  forms under either setting and gives bitwise the same result.
"""

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _both(ctx, fn):
    ctx.set_option("nl_bulk", -1)
    try:
        a = fn()
    finally:
        ctx.set_option("nl_bulk", 0)
    ctx.set_option("nl_bulk", 1)
    try:
        b = fn()
    finally:
        ctx.set_option("nl_bulk", 0)
    return a, b


@pytest.mark.parametrize("precision,tol", [("f64", 1e-14), ("f32", 2e-6)])
def test_bulk_forms_match_register_forms(precision, tol):
    import inq_b200 as ib
    from inq_b200 import synthetic
    prec = ib.F64 if precision == "f64" else ib.F32
    basis, ham, phi = synthetic.build(synthetic.config("c1", nst=32), precision=prec)
    a, b = _both(basis.ctx, lambda: ham(phi).matrix())
    assert np.linalg.norm(a - b) <= tol * np.linalg.norm(a)
    a, b = _both(basis.ctx, lambda: ib.exponential(ham, -0.05j, phi).matrix())
    assert np.linalg.norm(a - b) <= (1e-13 if prec == ib.F64 else tol) * np.linalg.norm(a)


def test_bulk_forms_with_overlapping_projectors(rng):
    import inq_b200 as ib
    from inq_b200 import pseudo
    r = np.linspace(0.0, 6.0, 601)
    beta_l, beta, cut = [], [], []
    for l in range(3):
        for k in range(2):
            rc = 1.3 + 0.2 * l + 0.1 * k
            bb = r ** l * np.exp(-(r / (0.5 * rc)) ** 2) * (1.0 + 0.3 * k * r)
            bb[r > rc] = 0.0
            beta_l.append(l)
            beta.append(bb)
            cut.append(int(np.searchsorted(r, rc)) + 1)
    d = np.zeros((6, 6))
    for i in range(6):
        for j in range(i, 6):
            if beta_l[i] == beta_l[j]:
                d[i, j] = d[j, i] = rng.uniform(-2, 2)
    ps = pseudo.Pseudopotential("Xx", 4.0, r, np.full_like(r, r[1] - r[0]), -2.0 * np.exp(-r ** 2), beta_l, beta, cut, d)
    lat = np.diag([8.0, 7.5, 8.5])
    sizes = (24, 20, 24)
    rs = ib.RealSpace(ib.Cell(lat), sizes=sizes)
    atoms = [(ps, np.array([1.0, 2.0, -1.5])), (ps, np.array([-3.0, 0.5, 2.5]))]
    points, pos, mats, coeff, npts, nlm, owner = pseudo.projector_tables(ib.Cell(lat), sizes, atoms)
    ham = ib.KSHamiltonian(rs)
    V = 0.3 * np.cos(2 * np.pi * np.arange(np.prod(sizes)) / 97.0).reshape(sizes)
    ham.set_scalar_potential(V)
    ham.set_projectors(points, pos, mats, coeff, npts, nlm)
    nst = 6
    x = rng.standard_normal(sizes + (nst,)) + 1j * rng.standard_normal(sizes + (nst,))
    kp = (0.1, -0.05, 0.2)
    phi = ib.OrbitalSet.from_array(rs, x, kpoint=kp)
    a, b = _both(rs.ctx, lambda: ham(phi).hypercubic())
    assert np.linalg.norm(a - b) <= 1e-14 * np.linalg.norm(a)
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
    ref = O.Hamiltonian(ors, V, O.ProjectorAll.pack(projs)).apply_real(x, kp)
    assert np.linalg.norm(b - ref) <= 1e-12 * np.linalg.norm(ref)


def test_odd_state_count_single_precision_takes_register_forms():
    import inq_b200 as ib
    from inq_b200 import synthetic
    basis, ham, phi = synthetic.build(synthetic.config("c1", nst=7), precision=ib.F32)
    a, b = _both(basis.ctx, lambda: ham(phi).matrix())
    assert np.array_equal(a, b)
