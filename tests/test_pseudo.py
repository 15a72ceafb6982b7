"""UPF pseudopotential reading and the projector tables built from it (CPU).

* The reader is pinned to the reference's projector test (projector.hpp:160-240): for its N.upf and
  N_non_diagonal.upf.gz files, 8 projector functions and the KB coefficients it checks (D_ij / 2,
  coupled only within equal m).  ``golden/upf_reference_pins.json`` holds what the reader parsed from
  those files (made by ``golden/make_upf_golden.py``); the KB coefficients are built from it on every
  run.  With INQ_REFERENCE_DATA naming the reference's unit-test data directory the files themselves
  are parsed again and compared with the pins.
* A synthetic UPF (version 2, written by ``write_upf``) reads back unchanged; a version-1 text
  block parses to the same values.
* Real spherical harmonics up to l = 3 are orthonormal on the sphere.
* The grouped projector tables (at most four functions per projector, coupled functions together)
  give the same dense nonlocal operator as the ungrouped functions with the full KB matrix.
"""

import os

import numpy as np
import pytest

from inq_b200 import pseudo

REF = os.environ.get("INQ_REFERENCE_DATA", "")
PINS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "upf_reference_pins.json")


def _pinned(name):
    import json
    with open(PINS) as f:
        p = json.load(f)[name]
    n = len(p["beta_l"])
    mesh = np.linspace(0.0, 1.0, 2)
    return pseudo.Pseudopotential(p["element"], p["z_valence"], mesh, mesh, mesh, list(p["beta_l"]),
                                  [mesh] * n, [1] * n, np.array(p["dij"]))


def _synthetic(lmax=2, nproj_per_l=2, seed=3):
    rng = np.random.default_rng(seed)
    r = np.linspace(0.0, 6.0, 601)
    rab = np.full_like(r, r[1] - r[0])
    beta_l, beta, cut = [], [], []
    for l in range(lmax + 1):
        for k in range(nproj_per_l):
            rc = 1.2 + 0.2 * l + 0.1 * k
            b = r ** l * np.exp(-(r / (0.5 * rc)) ** 2) * (1.0 + 0.3 * k * r)
            b[r > rc] = 0.0
            beta_l.append(l)
            beta.append(b)
            cut.append(int(np.searchsorted(r, rc)) + 1)
    nb = len(beta_l)
    d = np.zeros((nb, nb))
    for i in range(nb):
        for j in range(nb):
            if beta_l[i] == beta_l[j]:
                d[i, j] = d[j, i] = rng.uniform(-2, 2) if i != j else rng.uniform(-4, 4)
    vloc = -3.0 * np.exp(-r ** 2) - 1.0 / np.maximum(r, 1e-3) * (1 - np.exp(-r))
    return pseudo.Pseudopotential("Xx", 5.0, r, rab, vloc, beta_l, beta, cut, d)


def test_kb_coefficients_of_the_reference_projector_test():
    ps = _pinned("N.upf")
    assert ps.num_projectors_lm() == 8 and ps.z_valence == 5.0
    kb = ps.kb_coefficients()
    expect = [7.494508815, 0.6363049519, -4.2939052122, -4.2939052122, -4.2939052122,
              -1.0069878791, -1.0069878791, -1.0069878791]
    assert np.allclose(np.diag(kb), expect, atol=5e-10)
    assert np.count_nonzero(kb - np.diag(np.diag(kb))) == 0
    nd = _pinned("N_non_diagonal.upf.gz").kb_coefficients()
    assert nd[0, 0] == pytest.approx(4.0654068834, abs=5e-10) and nd[1, 1] == pytest.approx(4.0654068834, abs=5e-10)
    assert nd[0, 1] == pytest.approx(-3.4291019316, abs=5e-10) and nd[1, 0] == pytest.approx(-3.4291019316, abs=5e-10)
    for i in (2, 3, 4):
        assert nd[i, i] == pytest.approx(-2.6504465456, abs=5e-10)
        assert nd[i, i + 3] == pytest.approx(1.6434586665, abs=5e-10)
        assert nd[i + 3, i] == pytest.approx(1.6434586665, abs=5e-10)
    assert nd[0, 2] == 0.0 and nd[2, 3] == 0.0


def test_version_one_file_of_the_reference_data():
    ps = _pinned("F.UPF")
    assert ps.element == "F" and ps.z_valence == 7.0 and ps.beta_l == [0]


@pytest.mark.skipif(not (REF and os.path.exists(os.path.join(REF, "N.upf"))), reason="reference test data not given")
def test_reader_reproduces_the_pins():
    import json
    with open(PINS) as f:
        pins = json.load(f)
    for name, p in pins.items():
        ps = pseudo.read_upf(os.path.join(REF, name))
        assert ps.element == p["element"] and ps.z_valence == p["z_valence"] and ps.beta_l == p["beta_l"]
        assert np.array_equal(ps.dij, np.array(p["dij"])) and len(ps.r) == p["mesh_size"]
        assert ps.projector_radius() == p["projector_radius"] and ps.projector_radius() > 0.0


def test_write_and_read_back(tmp_path):
    ps = _synthetic()
    f = str(tmp_path / "x.upf")
    pseudo.write_upf(f, ps)
    q = pseudo.read_upf(f)
    assert q.element == "Xx" and q.z_valence == 5.0 and q.beta_l == ps.beta_l
    assert np.array_equal(q.r, ps.r) and np.allclose(q.vlocal, ps.vlocal, rtol=1e-15, atol=0)
    for a, b in zip(q.beta, ps.beta):
        assert np.allclose(a[1:], b[1:], rtol=1e-14, atol=1e-300)
    assert np.allclose(q.dij, ps.dij, rtol=1e-15, atol=0)
    assert q.num_projectors_lm() == 18


def test_version_one_text_block():
    txt = """<PP_INFO>
x
</PP_INFO>
<PP_HEADER>
   0                   Version Number
  Xx                   Element
   NC                  Norm - Conserving pseudopotential
    F                  Nonlinear Core Correction
 SLA  PW   NOGX NOGC   PZ   Exchange-Correlation functional
    3.00000000000      Z valence
    0.00000000000      Total energy
    0.0000000    0.0000000 Suggested cutoff for wfc and rho
    0                  Max angular momentum component
    4                  Number of points in mesh
    1    1             Number of Wavefunctions, Number of Projectors
</PP_HEADER>
<PP_MESH>
  <PP_R>
  0.0 0.5 1.0 1.5
  </PP_R>
  <PP_RAB>
  0.5 0.5 0.5 0.5
  </PP_RAB>
</PP_MESH>
<PP_LOCAL>
  -2.0 -1.0 -0.5 -0.25
</PP_LOCAL>
<PP_NONLOCAL>
  <PP_BETA>
    1    0             Beta    L
     3
  0.0 0.25 0.5
  </PP_BETA>
  <PP_DIJ>
    1                  Number of nonzero Dij
    1    1  3.0
  </PP_DIJ>
</PP_NONLOCAL>
"""
    import tempfile
    with tempfile.NamedTemporaryFile("w", suffix=".UPF", delete=False) as f:
        f.write(txt)
    try:
        ps = pseudo.read_upf(f.name)
    finally:
        os.unlink(f.name)
    assert ps.element == "Xx" and ps.z_valence == 3.0 and ps.beta_l == [0]
    assert np.allclose(ps.vlocal, [-1.0, -0.5, -0.25, -0.125])
    assert np.allclose(ps.beta[0][1:3], [0.5, 0.5])
    assert ps.dij[0, 0] == 1.5


def test_real_harmonics_are_orthonormal():
    # Gauss-Legendre in cos(theta) times a uniform phi grid integrates products of degree <= 6 exactly
    x, w = np.polynomial.legendre.leggauss(16)
    phi = np.arange(32) * (2 * np.pi / 32)
    ct, ph = np.meshgrid(x, phi, indexing="ij")
    st = np.sqrt(1 - ct ** 2)
    xyz = np.stack([st * np.cos(ph), st * np.sin(ph), ct], axis=-1).reshape(-1, 3)
    wt = (w[:, None] * np.full((1, 32), 2 * np.pi / 32)).reshape(-1)
    Y = np.concatenate([pseudo.real_ylm(l, 2.5 * xyz) for l in range(4)])
    G = (Y * wt) @ Y.T
    assert np.allclose(G, np.eye(16), atol=1e-12)


def test_groups_keep_coupled_functions_together():
    ps = _synthetic(lmax=3, nproj_per_l=2)
    groups = pseudo.group_functions(ps)
    assert sorted(sum(groups, [])) == list(range(ps.num_projectors_lm()))
    assert all(len(g) <= 4 for g in groups)
    fn = ps.lm_functions()
    kb = ps.kb_coefficients()
    where = {k: gi for gi, g in enumerate(groups) for k in g}
    for a in range(len(fn)):
        for b in range(len(fn)):
            if kb[a, b] != 0.0:
                assert where[a] == where[b]


def test_grouped_tables_give_the_full_nonlocal_operator():
    from inq_b200 import core
    ps = _synthetic(lmax=2, nproj_per_l=2)
    cell = core.Cell(np.diag([9.0, 8.0, 8.5]))
    sizes = (18, 16, 17)
    atoms = [(ps, np.array([1.0, 2.0, -1.5])), (ps, np.array([-3.0, 0.5, 2.0]))]
    points, pos, mats, coeff, npts, nlm, owner = pseudo.projector_tables(cell, sizes, atoms)
    assert len(points) == 2 * 5 and list(owner) == [0] * 5 + [1] * 5
    npoint = int(np.prod(sizes))
    # grouped: sum over projectors of P^T C P
    Vg = np.zeros((npoint, npoint))
    for p in range(len(points)):
        n = npts[p]
        flat = (points[p, :n, 0] * sizes[1] + points[p, :n, 1]) * sizes[2] + points[p, :n, 2]
        P = np.zeros((4, npoint))
        np.add.at(P.T, flat, mats[p, :, :n].T)
        Vg += P.T @ coeff[p] @ P
    # ungrouped: all functions of an atom with the full KB matrix
    Vf = np.zeros((npoint, npoint))
    for ps_, R in atoms:
        pts, dist, rel = core.spherical_grid(cell, sizes, R, ps_.projector_radius())
        xyz = rel.astype(np.float64) @ cell.lattice
        rows = []
        for i, l in enumerate(ps_.beta_l):
            rad = pseudo._radial(ps_, i, dist.astype(np.float64))
            for y in pseudo.real_ylm(l, xyz):
                rows.append(rad * y)
        flat = (pts[:, 0] * sizes[1] + pts[:, 1]) * sizes[2] + pts[:, 2]
        P = np.zeros((len(rows), npoint))
        np.add.at(P.T, flat, np.array(rows).T)
        Vf += P.T @ ps_.kb_coefficients() @ P
    assert np.allclose(Vg, Vf, rtol=0, atol=1e-12 * np.max(np.abs(Vf)))
    assert np.max(np.abs(Vf)) > 0


def _erf_pseudo(Z, a):
    from scipy.special import erf
    r = np.linspace(0, 12, 4001)
    v = np.where(r > 0, -Z * erf(r / a) / np.where(r > 0, r, 1), -Z * 2 / (np.sqrt(np.pi) * a))
    return pseudo.Pseudopotential("Xx", Z, r, np.full_like(r, r[1]), v)


def test_local_potential_does_not_depend_on_the_range_split():
    """V_loc = -Z erf(r/a)/r: the sphere part vanishes when sigma = a, and any other split gives the
    same grid potential; the grid average is alpha_Z / Omega = pi Z a^2 / Omega."""
    from inq_b200 import core
    cell = core.Cell(np.diag([7.0, 8.0, 7.5]))
    sizes = (28, 32, 30)
    for a in (0.8, 1.2):
        ps = _erf_pseudo(3.0, a)
        atoms = [(ps, np.array([0.3, -1.0, 0.7])), (ps, np.array([-2.0, 2.5, 1.0]))]
        v_auto = pseudo.local_potential(cell, sizes, atoms)
        v_a = pseudo.local_potential(cell, sizes, atoms, sigma=a)
        assert np.max(np.abs(v_auto - v_a)) < 1e-6 * np.max(np.abs(v_a))
        assert np.mean(v_a) == pytest.approx(2 * np.pi * 3.0 * a * a / cell.volume, rel=1e-12)


@pytest.mark.skipif(not (REF and os.path.exists(os.path.join(REF, "N.upf"))), reason="reference test data not given")
def test_local_potential_average_of_a_pseudopotential_file():
    """The grid average of the local potential of a real pseudopotential is its alpha_Z / Omega,
    alpha_Z = int (V_loc(r) + Z / r) 4 pi r^2 dr on the radial mesh."""
    from inq_b200 import core
    ps = pseudo.read_upf(os.path.join(REF, "N.upf"))
    cell = core.Cell(np.eye(3) * 10.0)
    v = pseudo.local_potential(cell, (40, 40, 40), [(ps, np.zeros(3))])
    r = ps.r
    f = (ps.vlocal + ps.z_valence / np.where(r > 0, r, 1.0)) * 4 * np.pi * r * r
    alpha = np.sum(0.5 * (f[1:] + f[:-1]) * np.diff(r))
    assert np.mean(v) == pytest.approx(alpha / cell.volume, rel=2e-3)
    assert np.isfinite(v).all()
