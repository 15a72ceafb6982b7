"""Real-time propagation driver and its results files (real_time/propagate.hpp, real_time/results.hpp).

``propagate`` steps a set of orbitals with ETRS (:func:`inq_b200.core.etrs`) and hands every step's
observables to ``Results``, which keeps the time series and writes them in the reference's
``real-time/observables`` layout (results.hpp:77-100, utils/load_save.hpp): text files
``total_steps``, ``total_time`` (one value each), ``time`` and ``total_energy`` (one value per line)
and ``dipole`` (three tab-separated values per line), numbers printed with 25 significant digits as a
C++ stream with ``precision(25)`` prints them.  Empty series are not written (their file is removed).
"""

from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np

from . import core


def _num(x: float) -> str:
    """A double as ``std::ostream << x`` prints it with precision 25 (default float notation)."""
    return f"{float(x):.25g}"


@dataclass
class Results:
    """real_time::results: per-step time, total energy and dipole."""
    total_steps: int = 0
    total_time: float = 0.0
    time: list = field(default_factory=list)
    total_energy: list = field(default_factory=list)
    dipole: list = field(default_factory=list)
    current: list = field(default_factory=list)

    def record(self, step: int, t: float, energy: float, dipole=None):
        """results::operator() (results.hpp:30-45) for one step's observables."""
        self.total_steps = int(step)
        self.total_time = float(t)
        self.time.append(float(t))
        self.total_energy.append(float(energy))
        if dipole is not None:
            self.dipole.append([float(v) for v in dipole])

    def save(self, dirname: str):
        """results::save (results.hpp:77-88)."""
        os.makedirs(dirname, exist_ok=True)
        with open(os.path.join(dirname, "total_steps"), "w") as f:
            f.write(f"{self.total_steps}\n")
        with open(os.path.join(dirname, "total_time"), "w") as f:
            f.write(_num(self.total_time) + "\n")
        for name, rows, fmt in (("time", self.time, _num), ("total_energy", self.total_energy, _num),
                                ("dipole", self.dipole, lambda v: "\t".join(_num(c) for c in v)),
                                ("current", self.current, lambda v: "\t".join(_num(c) for c in v))):
            path = os.path.join(dirname, name)
            if not rows:
                if os.path.exists(path):
                    os.remove(path)
                continue
            with open(path, "w") as f:
                for r in rows:
                    f.write(fmt(r) + "\n")

    @staticmethod
    def load(dirname: str) -> "Results":
        """results::load (results.hpp:90-105)."""
        res = Results()
        with open(os.path.join(dirname, "total_steps")) as f:
            res.total_steps = int(f.read().split()[0])
        with open(os.path.join(dirname, "total_time")) as f:
            res.total_time = float(f.read().split()[0])
        with open(os.path.join(dirname, "time")) as f:
            res.time = [float(v) for v in f.read().split()][: res.total_steps + 1]
        with open(os.path.join(dirname, "total_energy")) as f:
            res.total_energy = [float(v) for v in f.read().split()][: res.total_steps + 1]
        for name in ("dipole", "current"):
            path = os.path.join(dirname, name)
            if os.path.exists(path):
                with open(path) as f:
                    rows = [[float(c) for c in line.split()] for line in f if line.strip()]
                setattr(res, name, rows)
        return res


def band_energy(ham: core.KSHamiltonian, phis: Sequence[core.OrbitalSet], occupations: Sequence) -> float:
    """sum_s f_s <psi_s|H|psi_s> / <psi_s|psi_s>: the total energy of the fixed (non-interacting) Hamiltonian."""
    e = 0.0
    for phi, occ in zip(phis, occupations):
        eig, _ = ham.eigenvalues(phi)
        e += float(np.dot(np.asarray(occ, dtype=np.float64), eig))
    return e


def propagate(ham: core.KSHamiltonian, phis: Sequence[core.OrbitalSet], occupations: Sequence, dt: float,
              num_steps: int, results: Results | None = None, energy: Callable | None = None,
              every_energy: int = 1) -> Results:
    """real_time::propagate (propagate.hpp:87-119) with the ETRS step: the observables of the initial
    state (step 0) and of every step go to ``results``; ``energy(ham, phis, occupations)`` gives the
    total energy (default: the band energy of the fixed Hamiltonian, formed every ``every_energy``
    steps and repeated in between)."""
    res = results if results is not None else Results()
    energy = energy or band_energy
    dens = core.density(phis, occupations)
    basis = phis[0].basis
    e = energy(ham, phis, occupations)
    res.record(0, 0.0, e, core.dipole(basis, dens))
    for step in range(1, num_steps + 1):
        dens, dip, _ = core.etrs(ham, phis, occupations, dt, want_density=False)
        if step % every_energy == 0:
            e = energy(ham, phis, occupations)
        res.record(step, step * dt, e, dip)
    return res
