"""GPU tests of the batched execution and the serving loop.

* Batched H|psi> over uneven systems (the C4 construction) -- eager fork/join and the
  replayed CUDA graph -- gives bitwise the per-system results.
* The autotuner returns options the batch then uses, with unchanged results; per-Hamiltonian option
  overrides change only their own Hamiltonian's kernels.
* The serving loop returns, for every request, the same result alone and in a mix of
  concurrent requests (continuous batching over several streams).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def systems():
    import inq_b200 as ib
    from inq_b200 import synthetic
    sy = synthetic.batch_systems(10, max_states=64)
    out = []
    for s in sy:
        basis, ham, phi = synthetic.build(s, precision=ib.F32)
        out.append((s, basis, ham, phi))
    return out


def test_batch_eager_and_graph_match_individual(systems):
    from inq_b200.batch import Batch
    ctx = systems[0][1].ctx
    hams = [t[2] for t in systems]
    ins = [t[3] for t in systems]
    ref = []
    for h, p in zip(hams, ins):
        ref.append(h(p).matrix())
    outs = [p.skeleton() for p in ins]
    b = Batch(ctx, hams, ins, outs, nstreams=4)
    b.apply()
    ctx.synchronize()
    for r, o in zip(ref, outs):
        assert np.array_equal(r, o.matrix())
    for o in outs:
        o.fill(0.0)
    b.capture()
    b.launch()
    ctx.synchronize()
    for r, o in zip(ref, outs):
        assert np.array_equal(r, o.matrix())
    b.launch()  # replay again
    ctx.synchronize()
    for r, o in zip(ref, outs):
        assert np.array_equal(r, o.matrix())
    b.close()


def test_autotuned_batch(systems):
    from inq_b200.batch import Batch, autotune
    ctx = systems[0][1].ctx
    pairs = [(t[2], t[3]) for t in systems[:4]]
    tuning = autotune(pairs, reps=2)
    assert len(tuning.table) >= 1
    for opts in tuning.table.values():
        assert opts["fft_impl"] in (0, 1)
    hams = [p[0] for p in pairs]
    ins = [p[1] for p in pairs]
    ref = [h(p).matrix() for h, p in pairs]
    outs = [p.skeleton() for p in ins]
    b = Batch(ctx, hams, ins, outs, nstreams=2, tuning=tuning)
    b.apply()
    ctx.synchronize()
    # the tuned options live on each Hamiltonian: one batched call gives bitwise the individual applies
    for r, o in zip(ref, outs):
        assert np.array_equal(r, o.matrix())
    for h in hams:
        for k in tuning.table[next(iter(tuning.table))]:
            h.set_option(k, -1 if k != "nl_bulk" else 0)


def test_hamiltonian_option_overrides(systems):
    """inqb_hamiltonian_set_option: an override changes the kernels of that Hamiltonian's applications only
    (the generic FFT kernel and register-held nonlocal kernels give the same operator to rounding), and a
    negative value removes it."""
    import inq_b200 as ib
    s, basis, ham, phi = systems[0]
    other_s, other_basis, other_ham, other_phi = systems[1]
    ctx = basis.ctx
    ref = ham(phi).matrix()
    ref_other = other_ham(other_phi).matrix()
    n0 = ctx.launch_count()
    ham(phi)
    launches_default = ctx.launch_count() - n0
    ham.set_option("fft_impl", 1)
    ham.set_option("nl_bulk", -1)
    try:
        got = ham(phi).matrix()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-6
        # the other system (same context) keeps the context's options: bitwise its earlier result
        assert np.array_equal(other_ham(other_phi).matrix(), ref_other)
    finally:
        ham.set_option("fft_impl", -1)
        ham.set_option("nl_bulk", 0)
    assert np.array_equal(ham(phi).matrix(), ref)
    # fewer SMs for the persistent kernels: the same tiles, computed the same way
    ham.set_option("grid_sms", 16)
    try:
        assert np.array_equal(ham(phi).matrix(), ref)
    finally:
        ham.set_option("grid_sms", -1)
    with pytest.raises(ib.InqbError):
        ham.set_option("grid_sms", 100000)
    # another number of projection ranges per sphere sums the projections in another order
    ham.set_option("nl_project_ranges", 24)
    try:
        got = ham(phi).matrix()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-6
    finally:
        ham.set_option("nl_project_ranges", -1)
    assert np.array_equal(ham(phi).matrix(), ref)
    n0 = ctx.launch_count()
    ham(phi)
    assert ctx.launch_count() - n0 == launches_default
    with pytest.raises(ib.InqbError):
        ham.set_option("stream_priority", 1)


def test_serving_alone_equals_mix(systems):
    import inq_b200 as ib
    from inq_b200 import serving
    payloads = [serving.Payload(t[0], t[0].local_potential().reshape(-1), t[3].matrix()) for t in systems[:5]]
    def requests(spacing):
        rq = []
        for i, p in enumerate(payloads):
            rq.append(serving.Request(2 * i, "apply", p, arrival=spacing * 2 * i))
            rq.append(serving.Request(2 * i + 1, "etrs", p, steps=2, arrival=spacing * (2 * i + 1)))
        return rq
    alone = requests(0.0)
    srv = serving.Server(slots=1, precision=ib.F32, budget_bytes=8 << 30)
    st1 = srv.run(alone, realtime=False)
    srv.close()
    mix = requests(0.0)
    srv = serving.Server(slots=4, precision=ib.F32, budget_bytes=8 << 30)
    st2 = srv.run(mix, realtime=False)
    srv.close()
    assert st1["completed"] == st2["completed"] == len(alone)
    for a, m in zip(sorted(alone, key=lambda r: r.rid), sorted(mix, key=lambda r: r.rid)):
        assert not a.error and not m.error, (a.error, m.error)
        if a.kind == "apply":
            assert np.array_equal(a.result["hphi"], m.result["hphi"])
        else:
            assert np.array_equal(a.result["dipoles"], m.result["dipoles"])
            assert np.array_equal(a.result["phi"], m.result["phi"])
    assert st2["p99_ms"] >= st2["p50_ms"] > 0
