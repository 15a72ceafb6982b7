"""CPU-side checks of the C ABI: the library loads, exports every declared entry
point, reports errors as status codes, and its host sphere construction matches
the oracle bit for bit (spherical_grid.hpp:59-160)."""

import math
import os
import re

import numpy as np
import pytest

import oracle as O
from inq_b200 import _lib
from inq_b200 import core

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^\s*(?:int|const char \*)\s*(inqb_[a-z0-9_]+)\s*\(", txt, re.M))
    return names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    decl = declared_symbols()
    assert len(decl) >= 45
    missing = [n for n in sorted(decl) if not hasattr(lib, n)]
    assert not missing, missing
    # every declared entry point has a ctypes signature
    assert decl <= set(_lib.SIGNATURES), sorted(decl - set(_lib.SIGNATURES))


def test_error_codes_without_device():
    """No device here: creating a context must fail with a status, not crash."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(_lib.InqbError):
        core.Context(0)


def _compare_sphere(cell_lat, spacing, center, radius):
    ocell = O.Cell(cell_lat)
    rs = O.RealSpace.from_spacing(ocell, spacing)
    ref = O.spherical_grid(rs, np.array(center, dtype=float), radius)
    pts, dist, rel = core.spherical_grid(core.Cell(cell_lat), rs.sizes, center, radius)
    assert pts.shape == ref.points.shape
    assert np.array_equal(pts, ref.points)
    assert np.array_equal(dist, ref.distance)
    assert np.array_equal(rel, ref.relpos)
    return len(pts), rs


@pytest.mark.parametrize("center", [(0.0, 0.0, 0.0), (-5.0, 0.0, 0.0), (5.0, 5.0, 5.0), (2.5, 2.5, 2.5),
                                    (1.234, -3.21, 4.4)])
def test_sphere_matches_oracle_cubic(center):
    n, rs = _compare_sphere(np.diag([10.0] * 3), 0.49672941, center, 2.0)
    if center != (1.234, -3.21, 4.4):
        assert n == 257  # spherical_grid.hpp:269-358


def test_sphere_matches_oracle_noncubic():
    lat = [[7.57325, 0.0, 0.0], [-3.78662, 6.55862, 0.0], [5.78917e-16, 1.00271e-15, 9.45443]]
    n, rs = _compare_sphere(lat, 0.405578, (3.78659, -2.18619, 1.65434), 5.71)
    assert n == 15963  # spherical_grid.hpp:382-397
    assert abs(n * rs.volume_element() / (4.0 / 3.0 * math.pi * 5.71 ** 3) - 1.0013282291) < 1e-9


def test_sphere_matches_oracle_synthetic_atoms():
    from inq_b200 import synthetic
    s = synthetic.config("c1")
    ocell = O.Cell(s.lattice)
    rs = O.RealSpace(ocell, s.sizes)
    for R in s.positions:
        ref = O.spherical_grid(rs, R, s.radius)
        pts, dist, rel = core.spherical_grid(core.Cell(s.lattice), s.sizes, R, s.radius)
        assert np.array_equal(pts, ref.points) and np.array_equal(dist, ref.distance)
        assert np.array_equal(rel, ref.relpos)
