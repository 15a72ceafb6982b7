"""Restart files in the reference's on-disk layout (operations/io.hpp, systems/electrons.hpp:323-380).

CPU part: the host-only writers and readers of plain arrays and field sets produce the reference's
file names (ten-digit, zero-padded, utils/num_str.hpp:16-20) and raw float64 contents, and read them
back.  GPU part: an orbital set saved by the library holds one complex128 file per state with the
state's values in grid order, loads back bitwise (double) or to single precision, and a set the test
writes itself in that layout loads into the library."""

import os

import numpy as np
import pytest

from inq_b200 import _lib


def test_array_and_field_layout(tmp_path):
    lib = _lib.load()
    occ = np.array([2.0, 2.0, 1.5, 0.0])
    d = str(tmp_path / "occupations")
    _lib.check(lib.inqb_array_save(d.encode(), _lib.dptr(occ), occ.size))
    assert os.listdir(d) == ["array"]
    assert np.array_equal(np.fromfile(os.path.join(d, "array"), dtype=np.float64), occ)
    back = np.zeros(4)
    _lib.check(lib.inqb_array_load(d.encode(), _lib.dptr(back), 4))
    assert np.array_equal(back, occ)
    rho = np.random.default_rng(1).random((60, 2))
    f = str(tmp_path / "spin_density")
    _lib.check(lib.inqb_field_save(f.encode(), _lib.dptr(np.ascontiguousarray(rho)), 60, 2))
    assert sorted(os.listdir(f)) == ["0000000000", "0000000001"]
    for c in range(2):
        assert np.array_equal(np.fromfile(os.path.join(f, f"{c:010d}"), dtype=np.float64), rho[:, c])
    got = np.zeros((60, 2))
    _lib.check(lib.inqb_field_load(f.encode(), _lib.dptr(got), 60, 2))
    assert np.array_equal(got, rho)


def test_missing_files_are_errors(tmp_path):
    lib = _lib.load()
    x = np.zeros(10)
    with pytest.raises(_lib.InqbError):
        _lib.check(lib.inqb_array_load(str(tmp_path / "nothing").encode(), _lib.dptr(x), 10))
    d = str(tmp_path / "short")
    _lib.check(lib.inqb_array_save(d.encode(), _lib.dptr(np.zeros(3)), 3))
    with pytest.raises(_lib.InqbError):
        _lib.check(lib.inqb_array_load(d.encode(), _lib.dptr(x), 10))


@pytest.mark.gpu
@pytest.mark.parametrize("precision_name", ["F64", "F32"])
def test_orbitals_save_load(tmp_path, rng, precision_name):
    import inq_b200 as ib
    prec = getattr(ib, precision_name)
    rs = ib.RealSpace(ib.Cell.cubic(8.0), sizes=(12, 10, 14))
    x = rng.standard_normal((12, 10, 14, 7)) + 1j * rng.standard_normal((12, 10, 14, 7))
    phi = ib.OrbitalSet.from_array(rs, x, precision=prec)
    d = str(tmp_path / "states")
    phi.save(d)
    names = sorted(os.listdir(d))
    assert names == [f"{s:010d}_{0:010d}" for s in range(7)]
    m = phi.matrix()
    for s in range(7):
        v = np.fromfile(os.path.join(d, names[s]), dtype=np.complex128)
        assert np.array_equal(v, m[:, s].astype(np.complex128))
    back = ib.OrbitalSet(rs, 7, precision=prec).load(d)
    assert np.array_equal(back.matrix(), m)
    # a set written in the layout by hand loads into the library
    d2 = str(tmp_path / "by_hand")
    os.makedirs(d2)
    y = rng.standard_normal((rs.size(), 7)) + 1j * rng.standard_normal((rs.size(), 7))
    for s in range(7):
        y[:, s].astype(np.complex128).tofile(os.path.join(d2, f"{s:010d}_{0:010d}"))
    got = ib.OrbitalSet(rs, 7, precision=ib.F64).load(d2)
    assert np.array_equal(got.matrix(), y)


@pytest.mark.gpu
def test_electrons_restart_round_trip(tmp_path, rng):
    import inq_b200 as ib
    rs = ib.RealSpace(ib.Cell.cubic(8.0), sizes=(12, 12, 12))
    x = rng.standard_normal((12, 12, 12, 5)) + 1j * rng.standard_normal((12, 12, 12, 5))
    phi = ib.OrbitalSet.from_array(rs, x)
    occ = np.array([2.0, 2.0, 2.0, 1.0, 0.0])
    dens = ib.density([phi], [occ])
    ib.save_electrons(str(tmp_path / "restart"), [phi], [occ], dens)
    assert os.path.isdir(tmp_path / "restart" / "kpin0000000000" / "states")
    other = ib.OrbitalSet(rs, 5)
    occs, d = ib.load_electrons(str(tmp_path / "restart"), [other])
    assert np.array_equal(other.matrix(), phi.matrix())
    assert np.array_equal(occs[0], occ)
    assert np.array_equal(d[:, 0], np.asarray(dens).reshape(-1))
