"""inq_b200: the Kohn-Sham H|psi> path of LLNL/inq, rebuilt for NVIDIA B200 (sm_100a).

The compute runs in libinqb200.so (hand-written CUDA behind the C ABI of
include/inqb.h); this package is its Python host interface, named after the
reference's C++ types (see :mod:`inq_b200.core`).
"""

from ._lib import F32, F64, FOURIER_SPACE, REAL_SPACE, InqbError  # noqa: F401
from .core import (  # noqa: F401
    Cell, Context, FourierSpace, Kick, KSHamiltonian, OrbitalSet, RealSpace, apply_phase_kick, cholesky_inverse, density,
    device_alloc_count,
    dipole, etrs, exponential, exponential_2_for_1, exponential_in_place, hermitian_eigen, laplacian, load_electrons,
    orthogonalize, overlap, overlap_diagonal, rotate, rotate_to, save_electrons, shift, spherical_grid, to_fourier, to_real)

__all__ = [n for n in dir() if not n.startswith("_")]
