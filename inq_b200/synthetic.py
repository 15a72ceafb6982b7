"""Seeded synthetic systems for the benchmark configurations.

The reference measures on real pseudopotential systems that need data files and
absent submodules; these configurations stand in for them with the same shapes:

* C1 ``c1``  cubic a = 10.26 bohr, 32^3 grid, 16 orbitals, 8 atoms on diamond sites;
* C2 ``c2``  a = 20.52, 96^3, 256 orbitals, 64 atoms (2x2x2 diamond supercell),
  positions jittered N(0, 0.05 bohr);
* C3 ``c3``  a = 25.6, 120^3, 256 orbitals, 128 atoms (diamond sites of a 2x2x4
  arrangement of conventional cells mapped into the cubic cell), jittered;
* C4 ``batch`` 64 systems, grids from {24,32,40,48,64,72}^3, 8-128 orbitals, 2-32 atoms.

Every system has: V_loc = sum_atoms -2 exp(-|r - R|^2 / 1 bohr^2) (minimum image,
float64); one Kleinman-Bylander projector set per atom with l = 0, 1 (nlm = 4),
radial exp(-r^2/rc^2), rc = 2 bohr, on the sphere |r - R| <= 2 bohr; a symmetric 4x4
KB coefficient matrix per atom with entries U[-1, 1]; orbitals with N(0,1)+iN(0,1)
Fourier coefficients for |G|^2/2 < ecut = 25 Ha, transformed to real space and
Cholesky-orthonormalised in FP64 on the device.

Random numbers come from SplitMix64 counter streams (Steele, Lea & Flood 2014) with
Box-Muller normals, so every quantity is a pure function of (seed, index).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)

SPHERE_RADIUS = 2.0   # bohr: projector sphere radius (generator constant)
RC = 2.0              # bohr: Gaussian radial width
ECUT = 25.0           # Ha
V_DEPTH = -2.0        # Ha
V_WIDTH = 1.0         # bohr

# stream offsets within one seed
STREAM_JITTER = 1
STREAM_KB = 2
STREAM_BATCH = 3


def splitmix64(seed: int, counters: np.ndarray) -> np.ndarray:
    c = np.asarray(counters, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed & (2 ** 64 - 1)) + (c + np.uint64(1)) * GOLDEN
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, counters) -> np.ndarray:
    return (splitmix64(seed, counters) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """n standard normals from counters offset.. (Box-Muller on pairs)."""
    m = (n + 1) // 2
    c = np.arange(offset, offset + 2 * m, dtype=np.uint64)
    u = uniform(seed, c).reshape(m, 2)
    r = np.sqrt(-2.0 * np.log(1.0 - u[:, 0]))
    z = np.stack([r * np.cos(2.0 * math.pi * u[:, 1]), r * np.sin(2.0 * math.pi * u[:, 1])], axis=1).reshape(-1)
    return z[:n]


def diamond_fractional():
    fcc = np.array([[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0]])
    return np.concatenate([fcc, fcc + 0.25])


def diamond_sites(reps=(1, 1, 1)):
    """Fractional coordinates (in the supercell) of the diamond sites of reps conventional cells."""
    base = diamond_fractional()
    out = []
    for i in range(reps[0]):
        for j in range(reps[1]):
            for k in range(reps[2]):
                out.append((base + np.array([i, j, k])) / np.array(reps, dtype=float))
    return np.concatenate(out)


@dataclass
class System:
    name: str
    lattice: np.ndarray            # [3,3] rows
    sizes: tuple
    nst: int
    positions: np.ndarray          # [natoms,3] cartesian
    kb: np.ndarray                 # [natoms,4,4]
    seed: int
    radius: float = SPHERE_RADIUS
    rc: float = RC
    ecut: float = ECUT
    meta: dict = field(default_factory=dict)

    @property
    def natoms(self):
        return len(self.positions)

    @property
    def npoints(self):
        return int(np.prod(self.sizes))

    def local_potential(self) -> np.ndarray:
        """V_loc [nx,ny,nz] = sum_a -2 exp(-|r - R_a|^2), minimum image in fractional coordinates."""
        lat = self.lattice
        inv = np.linalg.inv(lat)                 # cart = frac @ lat  ->  frac = cart @ inv
        axes = [np.arange(n) / n for n in self.sizes]
        frac_pos = self.positions @ inv
        V = np.zeros(self.sizes)
        for fa in frac_pos:
            d = [axes[k][:, None, None] if k == 0 else (axes[k][None, :, None] if k == 1 else axes[k][None, None, :])
                 for k in range(3)]
            dd = [d[k] - fa[k] for k in range(3)]
            dd = [x - np.round(x) for x in dd]
            # cartesian |dd @ lat|^2
            r2 = np.zeros(self.sizes)
            for j in range(3):
                comp = dd[0] * lat[0, j] + dd[1] * lat[1, j] + dd[2] * lat[2, j]
                r2 = r2 + comp * comp
            V += V_DEPTH * np.exp(-r2 / (V_WIDTH * V_WIDTH))
        return V


def _kb_matrices(seed: int, natoms: int) -> np.ndarray:
    u = uniform(seed + STREAM_KB, np.arange(natoms * 16, dtype=np.uint64)).reshape(natoms, 4, 4)
    k = 2.0 * u - 1.0
    return np.triu(k) + np.transpose(np.triu(k, 1), (0, 2, 1))


def make_system(name: str, a: float, n: int, nst: int, frac_sites: np.ndarray, seed: int,
                jitter: float = 0.0) -> System:
    lat = np.diag([a, a, a]).astype(np.float64)
    pos = frac_sites @ lat
    if jitter > 0.0:
        pos = pos + jitter * normal(seed + STREAM_JITTER, pos.size).reshape(pos.shape)
    return System(name, lat, (n, n, n), nst, pos, _kb_matrices(seed, len(pos)), seed)


def config(name: str, seed: int = 20240601, nst: int | None = None, n: int | None = None) -> System:
    """The named configuration; ``nst`` / ``n`` override the state count / grid (tests use smaller ones)."""
    if name == "c1":
        return make_system("c1", 10.26, n or 32, nst or 16, diamond_sites((1, 1, 1)), seed)
    if name == "c2":
        return make_system("c2", 20.52, n or 96, nst or 256, diamond_sites((2, 2, 2)), seed, jitter=0.05)
    if name == "c3":
        return make_system("c3", 25.6, n or 120, nst or 256, diamond_sites((2, 2, 4)), seed, jitter=0.05)
    raise ValueError(f"unknown configuration {name}")


def max_kinetic_energy(sysm: System) -> float:
    """Largest kinetic energy 1/2 |G|^2 (Ha) on the system's grid: the corners of the symmetric G range."""
    rec = 2.0 * np.pi * np.linalg.inv(sysm.lattice).T     # rows: reciprocal vectors b_i (a_i . b_j = 2 pi delta_ij)
    half = np.array(sysm.sizes, dtype=np.float64) / 2.0
    best = 0.0
    for sx in (-1, 1):
        for sy in (-1, 1):
            for sz in (-1, 1):
                g = (np.array([sx, sy, sz]) * half) @ rec
                best = max(best, 0.5 * float(g @ g))
    return best


def taylor_stable_dt(sysm: System, margin: float = 0.5) -> float:
    """A time step at which the order-4 Taylor propagator (exponential.hpp:21-69) stays bounded.

    |sum_{n<=4} (-i x)^n / n!|^2 = 1 - x^6/72 + x^8/576 exceeds 1 for x = dt * E > 2 sqrt(2), so
    the spectrum's top (the grid's largest kinetic energy) fixes dt < 2 sqrt(2) / E_max; ``margin``
    scales that bound."""
    return margin * 2.0 * np.sqrt(2.0) / max_kinetic_energy(sysm)


BATCH_GRIDS = (24, 32, 40, 48, 64, 72)


def batch_systems(count: int = 64, seed: int = 20240601, max_states: int = 128, min_states: int = 8,
                  min_atoms: int = 2, max_atoms: int = 32) -> list[System]:
    """C4: independent systems of uneven grid, state and atom counts (per-system seed = seed + index)."""
    out = []
    for i in range(count):
        s = seed + 1000 * (i + 1)
        u = uniform(seed + STREAM_BATCH, np.arange(3 * i, 3 * i + 3, dtype=np.uint64))
        n = BATCH_GRIDS[int(u[0] * len(BATCH_GRIDS)) % len(BATCH_GRIDS)]
        nst = min_states + int(u[1] * (max_states - min_states + 1))
        nat = min_atoms + int(u[2] * (max_atoms - min_atoms + 1))
        reps = 1
        while 8 * reps ** 3 < nat:
            reps += 1
        sites = diamond_sites((reps, reps, reps))[:nat]
        out.append(make_system(f"batch{i}", 10.26 * reps, n, nst, sites, s, jitter=0.05))
    return out


# ---------------------------------------------------------------- device construction


def build(sysm: System, precision=None, ctx=None):
    """Basis, Hamiltonian and orthonormal orbitals of a system on the device.

    Returns (basis, hamiltonian, orbitals in real space).  Orbitals are generated and
    orthonormalised in FP64; with precision F32 they are then converted."""
    from . import core
    from ._lib import F32, F64

    basis = core.RealSpace(core.Cell(sysm.lattice), sizes=sysm.sizes, ctx=ctx)
    ham = core.KSHamiltonian(basis)
    ham.set_scalar_potential(sysm.local_potential())
    ham.update_projectors_gaussian(sysm.positions, sysm.radius, sysm.rc, sysm.kb)
    fphi = core.OrbitalSet(basis, sysm.nst, space=core.FOURIER_SPACE, precision=F64)
    fphi.randomize_gsphere(sysm.seed, sysm.ecut)
    phi = core.to_real(fphi)
    del fphi
    core.orthogonalize(phi)
    if precision is not None and precision != F64:
        phi32 = phi.converted(F32)
        del phi
        return basis, ham, phi32
    return basis, ham, phi
