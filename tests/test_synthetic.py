"""The seeded synthetic-system generator: determinism and the configuration shapes."""

import numpy as np

from inq_b200 import synthetic


def test_splitmix_known_values():
    # SplitMix64 with seed 0: first outputs of the published generator (Vigna's splitmix64.c)
    z = synthetic.splitmix64(0, np.arange(3, dtype=np.uint64))
    assert [int(x) for x in z] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_normals_are_standard():
    x = synthetic.normal(7, 200000)
    assert abs(x.mean()) < 0.01 and abs(x.std() - 1.0) < 0.01


def test_configs_shapes_and_determinism():
    c1 = synthetic.config("c1")
    assert c1.sizes == (32, 32, 32) and c1.nst == 16 and c1.natoms == 8
    c2 = synthetic.config("c2")
    assert c2.sizes == (96, 96, 96) and c2.nst == 256 and c2.natoms == 64
    c3 = synthetic.config("c3")
    assert c3.sizes == (120, 120, 120) and c3.natoms == 128
    again = synthetic.config("c2")
    assert np.array_equal(c2.positions, again.positions) and np.array_equal(c2.kb, again.kb)
    # jitter is small and KB matrices are symmetric with entries in [-1, 1]
    base = synthetic.diamond_sites((2, 2, 2)) * 20.52
    assert np.max(np.abs(c2.positions - base)) < 0.5
    assert np.allclose(c2.kb, np.transpose(c2.kb, (0, 2, 1)))
    assert np.all(np.abs(c2.kb) <= 1.0)


def test_local_potential():
    c1 = synthetic.config("c1")
    V = c1.local_potential()
    assert V.shape == (32, 32, 32)
    assert V.min() < -1.9 and V.max() <= 0.0
    # an atom at the origin: V(0) = -2 (+ tiny tails of the others)
    assert abs(V[0, 0, 0] + 2.0) < 1e-3


def test_batch_systems():
    sy = synthetic.batch_systems(64)
    assert len(sy) == 64
    for s in sy:
        assert s.sizes[0] in synthetic.BATCH_GRIDS
        assert 8 <= s.nst <= 128 and 2 <= s.natoms <= 32
    assert len({s.sizes[0] for s in sy}) >= 4
