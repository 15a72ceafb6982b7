"""GPU test of the bounded device-side waits without a fault or a hang.

A kernel waits on an mbarrier phase that nothing completes; its wait runs out after 50 ms of
%globaltimer and raises the context's error flag, as an expired wait of the FFT ring, the tensor-core
overlap or the bulk-copy nonlocal kernels would.  The host reads the flag: the next synchronize
reports INQB_ERR_TIMEOUT (status 7) and clears it, and the context stays usable (an H application
afterwards equals one before)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_expired_wait_is_reported_and_the_context_stays_usable():
    import inq_b200 as ib
    from inq_b200 import _lib, synthetic
    basis, ham, phi = synthetic.build(synthetic.config("c1", nst=8))
    ctx = basis.ctx
    before = ham(phi).matrix()
    ctx.check_wait_timeout(0.05)
    with pytest.raises(_lib.InqbError) as e:
        ctx.synchronize()
    assert e.value.code == 7 and "time limit" in str(e.value)
    ctx.synchronize()                      # the flag was cleared
    assert np.array_equal(ham(phi).matrix(), before)
    ctx.synchronize()
    with pytest.raises(_lib.InqbError):
        ctx.check_wait_timeout(5.0)        # the limit is bounded by the ABI
