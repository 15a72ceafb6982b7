"""real_time::results files (results.hpp:77-105, utils/load_save.hpp): the layout the reference writes
and reads -- value files, one number per line, tab-separated dipoles, 25 significant digits -- and a
round trip; on the GPU, a short propagation records one entry per step."""

import os

import numpy as np
import pytest

from inq_b200.real_time import Results


def test_results_layout_and_round_trip(tmp_path):
    r = Results()
    for k in range(4):
        r.record(k, 0.05 * k, -12.5 + 1e-3 * k, [0.1 * k, -0.2, 1.0 / 3.0])
    d = str(tmp_path / "observables")
    r.save(d)
    assert sorted(os.listdir(d)) == ["dipole", "time", "total_energy", "total_steps", "total_time"]
    assert open(os.path.join(d, "total_steps")).read() == "3\n"
    assert open(os.path.join(d, "total_time")).read() == "0.1500000000000000222044605\n"  # 0.05 * 3
    lines = open(os.path.join(d, "dipole")).read().splitlines()
    assert len(lines) == 4 and lines[1].split("\t")[2] == "0.3333333333333333148296163"
    back = Results.load(d)
    assert back.total_steps == 3 and back.time == r.time and back.total_energy == r.total_energy
    assert np.array_equal(np.array(back.dipole), np.array(r.dipole))
    # an empty series removes its file
    r.dipole = []
    r.save(d)
    assert not os.path.exists(os.path.join(d, "dipole"))


@pytest.mark.gpu
def test_propagate_records_every_step(tmp_path):
    import inq_b200 as ib
    from inq_b200 import synthetic
    from inq_b200.real_time import propagate
    sysm = synthetic.config("c1", nst=8)
    basis, ham, phi = synthetic.build(sysm)
    ib.apply_phase_kick(phi, [0.01, 0.0, 0.0])
    occ = np.full(sysm.nst, 2.0)
    res = propagate(ham, [phi], [occ], synthetic.taylor_stable_dt(sysm), 3)
    assert res.total_steps == 3 and len(res.time) == 4 and len(res.dipole) == 4
    # the fixed Hamiltonian conserves the band energy to the propagator's accuracy
    assert max(abs(e - res.total_energy[0]) for e in res.total_energy) < 1e-6 * abs(res.total_energy[0])
    res.save(str(tmp_path / "obs"))
    assert Results.load(str(tmp_path / "obs")).total_steps == 3
