"""GPU tests of the context options a serving loop uses to place the work of several contexts.

* ``grid_sms`` sizes the persistent kernels' grids for fewer SMs: H|psi> and the overlap are
  bitwise the same (every tile is computed the same way whatever CTA takes it, and the overlap's
  reduction split follows the device's SM count, not the option).
* ``stream_priority`` replaces the context's stream after the work queued on it: results are
  bitwise the same, and the stream handle changes.
* Out-of-range values are refused.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(ib, rng):
    from inq_b200 import synthetic
    sysm = synthetic.config("c1", nst=32, n=32)
    basis, ham, phi = synthetic.build(sysm, precision=ib.F32)
    return basis, ham, phi


def test_grid_sms_and_priority_leave_results_unchanged(rng):
    import inq_b200 as ib
    basis, ham, phi = _setup(ib, rng)
    ctx = basis.ctx
    ref = ham(phi).matrix()
    ref_s = ib.overlap(phi)
    ctx.set_option("grid_sms", 37)
    try:
        assert np.array_equal(ham(phi).matrix(), ref)
        assert np.array_equal(ib.overlap(phi), ref_s)
    finally:
        ctx.set_option("grid_sms", 0)
    s0 = ctx.stream()
    ctx.set_option("stream_priority", 1)
    try:
        assert ctx.stream() != s0
        assert np.array_equal(ham(phi).matrix(), ref)
    finally:
        ctx.set_option("stream_priority", 0)
    assert np.array_equal(ham(phi).matrix(), ref)


def test_option_ranges_are_checked(rng):
    import inq_b200 as ib
    basis, _, _ = _setup(ib, rng)
    ctx = basis.ctx
    for key, bad in (("grid_sms", -1), ("grid_sms", 100000), ("stream_priority", 2)):
        with pytest.raises(ib.InqbError):
            ctx.set_option(key, bad)
