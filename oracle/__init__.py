"""CPU oracle for the Kohn-Sham H|psi> path (TEST INFRASTRUCTURE ONLY).

This package is a float64 numpy restatement of the reference's operator sequence
(LLNL/inq, header-only C++).  It exists so the tests, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` leg of ``bench.py`` can check the CUDA path.  Nothing in
the ``inq_b200`` package imports it, and the product path never falls back to it.

Parity pins (the reference's own known-answer tests, restated in
``tests/test_oracle_pins.py``):

* spherical_grid.hpp:258-399 -- sphere sizes 257 / 15963, volume ratios
  0.9586598525 / 1.0013282291;
* ks_hamiltonian.hpp:324-536 -- constant -> 0, plane wave -> k^2/2, harmonic
  oscillator mean deviation 0.0051420503 (real and Fourier forms);
* transform.hpp:273-415 -- Gaussian FT vs analytic, round trip, fs volume
  0.0293659268, zero_outside_sphere ratio 0.5240308896;
* laplacian.hpp:143-200 -- plane-wave Laplacian;
* exponential.hpp:89-140 -- exp of a diagonal operator;
* orthogonalize.hpp:72-130 -- S = I after Cholesky orthogonalisation.

The nonlocal projector path (projector_all.hpp) and ETRS time series have no
runnable known answer in the reference (they need pseudopotential files and the
absent pseudopod/boost-multi submodules): for those the restatement itself is
the oracle ("parity unpinned" for those two rows).
"""

from .inq_oracle import *  # noqa: F401,F403
