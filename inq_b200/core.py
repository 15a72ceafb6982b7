"""Python host interface of the B200 H|psi> path, named after the reference's C++ API.

The classes mirror the reference types a caller of ``ks_hamiltonian`` handles:

* :class:`Cell`          -- systems::cell (src/systems/cell.hpp:26-215)
* :class:`RealSpace`     -- basis::real_space (src/basis/real_space.hpp:25-230)
* :class:`FourierSpace`  -- basis::fourier_space (src/basis/fourier_space.hpp:24-140)
* :class:`OrbitalSet`    -- states::orbital_set (src/states/orbital_set.hpp:18-192)
* :class:`KSHamiltonian` -- hamiltonian::ks_hamiltonian (src/hamiltonian/ks_hamiltonian.hpp:35-275)

and the free functions of operations::transform, operations::overlap,
operations::orthogonalize, operations::exponential, observables::density /
dipole, perturbations::kick and real_time::etrs.  Every call goes through the
C ABI of libinqb200.so; arrays cross it as [npoint][nst] complex, the
reference's field_set::matrix() layout.
"""

from __future__ import annotations

import ctypes as C
import heapq
import math
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import DP, F32, F64, FOURIER_SPACE, REAL_SPACE, check, dptr

# ---------------------------------------------------------------- context


class Context:
    """One device, one stream (the C ABI's inqb_ctx)."""

    _default: dict = {}

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        code = self.lib.inqb_ctx_create(device, C.byref(h))
        if code != 0:
            msg = self.lib.inqb_last_error(None)
            raise _lib.InqbError(code, msg.decode() if msg else "")
        self.handle = h
        self.device = device

    @classmethod
    def default(cls, device: int = 0) -> "Context":
        if device not in cls._default:
            cls._default[device] = Context(device)
        return cls._default[device]

    def check(self, code):
        check(code, self.handle)

    def synchronize(self):
        self.check(self.lib.inqb_ctx_synchronize(self.handle))

    def check_wait_timeout(self, limit_s: float = 0.05):
        """Queue the bounded-wait self-test: the next ``synchronize`` raises InqbError (INQB_ERR_TIMEOUT)."""
        self.check(self.lib.inqb_ctx_check_wait_timeout(self.handle, int(limit_s * 1e9)))

    def stream(self) -> int:
        p = C.c_void_p()
        self.check(self.lib.inqb_ctx_stream(self.handle, C.byref(p)))
        return p.value or 0

    def launch_count(self) -> int:
        n = C.c_longlong()
        self.check(self.lib.inqb_ctx_launch_count(self.handle, C.byref(n)))
        return n.value

    def set_option(self, key: str, value: int):
        self.check(self.lib.inqb_ctx_set_option(self.handle, key.encode(), int(value)))

    def mem_info(self):
        f, t = C.c_size_t(), C.c_size_t()
        self.check(self.lib.inqb_ctx_mem_info(self.handle, C.byref(f), C.byref(t)))
        return f.value, t.value

    def close(self):
        if getattr(self, "handle", None):
            self.lib.inqb_ctx_destroy(self.handle)
            self.handle = None


def device_alloc_count() -> int:
    """Device allocations the library has made in this process so far (inqb_device_alloc_count)."""
    n = C.c_longlong()
    check(_lib.load().inqb_device_alloc_count(C.byref(n)))
    return n.value


# ---------------------------------------------------------------- cell and bases


def nextprod(factors, n):
    """Smallest product of powers of ``factors`` that is >= n (math/nextprod.hpp)."""
    if n <= 1:
        return 1
    heap = list(factors)
    heapq.heapify(heap)
    seen = set(heap)
    while heap:
        cur = heapq.heappop(heap)
        if cur >= n:
            return cur
        for f in factors:
            if cur * f not in seen:
                seen.add(cur * f)
                heapq.heappush(heap, cur * f)
    raise ValueError(n)


class Cell:
    """Lattice vectors as rows (cartesian bohr), systems::cell."""

    def __init__(self, lattice, periodicity: int = 3):
        self.lattice = np.ascontiguousarray(np.asarray(lattice, dtype=np.float64).reshape(3, 3))
        self.periodicity = periodicity
        a0, a1, a2 = self.lattice
        self.volume = float(np.dot(a0, np.cross(a1, a2)))
        if self.volume < 1e-10:
            raise ValueError("the lattice volume is not positive")
        self.reciprocal = 2.0 * math.pi / self.volume * np.array([np.cross(a1, a2), np.cross(a2, a0), np.cross(a0, a1)])

    @classmethod
    def cubic(cls, a):
        return cls(np.diag([a, a, a]))

    @classmethod
    def orthorhombic(cls, a, b, c):
        return cls(np.diag([a, b, c]))

    def lengths(self):
        return np.sqrt(np.sum(self.lattice ** 2, axis=1))

    # metric helpers (cell.hpp:146-215)
    def cov_to_cart(self, v):
        return (self.reciprocal / (2.0 * math.pi)).T @ np.asarray(v, dtype=np.float64)

    def cart_to_cov(self, v):
        return self.lattice @ np.asarray(v, dtype=np.float64)

    def cart_to_contra(self, v):
        return (self.reciprocal / (2.0 * math.pi)) @ np.asarray(v, dtype=np.float64)

    def contra_to_cart(self, v):
        return self.lattice.T @ np.asarray(v, dtype=np.float64)


class RealSpace:
    """basis::real_space on one device."""

    def __init__(self, cell: Cell, spacing: float | None = None, sizes: Sequence[int] | None = None,
                 ctx: Context | None = None):
        self.cell = cell
        if sizes is None:
            if spacing is None:
                raise ValueError("give a spacing or the grid sizes")
            sizes = [nextprod([2, 3, 5, 7], int(math.floor(l / spacing + 0.5))) for l in cell.lengths()]
        self.sizes = tuple(int(s) for s in sizes)
        self.ctx = ctx or Context.default()
        lib = self.ctx.lib
        h = C.c_void_p()
        self.ctx.check(lib.inqb_basis_create(self.ctx.handle, dptr(cell.lattice.reshape(-1).copy()), *self.sizes,
                                             C.byref(h)))
        self.handle = h

    def size(self) -> int:
        return self.sizes[0] * self.sizes[1] * self.sizes[2]

    def volume_element(self) -> float:
        return self.cell.volume / self.size()

    def rspacing(self):
        return self.cell.lengths() / np.array(self.sizes)

    def reciprocal(self) -> "FourierSpace":
        return FourierSpace(self)

    def rvector_contra(self):
        """[nx,ny,nz,3] contravariant point positions in the symmetric range (real_space.hpp:127-135)."""
        idx = [np.where(np.arange(n) >= (n + 1) // 2, np.arange(n) - n, np.arange(n)) * (1.0 / n) for n in self.sizes]
        X, Y, Z = np.meshgrid(*idx, indexing="ij")
        return np.stack([X, Y, Z], axis=-1)

    def rvector_cartesian(self):
        return self.rvector_contra() @ self.cell.lattice

    def __del__(self):
        try:
            if getattr(self, "handle", None) and self.ctx.handle:
                self.ctx.lib.inqb_basis_destroy(self.handle)
        except Exception:
            pass


class FourierSpace:
    """basis::fourier_space(real_space): same grid, serial (non-reversed) order."""

    def __init__(self, rs: RealSpace):
        self.real_space = rs
        self.sizes = rs.sizes
        self.cell = rs.cell

    def size(self):
        return self.real_space.size()

    def volume_element(self):
        return self.cell.volume / (self.size() * self.size())  # fourier_space.hpp:48-50


def spherical_grid(cell: Cell, sizes, center, radius):
    """basis::spherical_grid on the host: (points [n,3] int32, distance [n] float32, relpos [n,3] float32)."""
    lib = _lib.load()
    lat = np.ascontiguousarray(cell.lattice.reshape(-1))
    c = np.ascontiguousarray(center, dtype=np.float64)
    n = C.c_longlong()
    code = lib.inqb_spherical_grid(dptr(lat), *[int(x) for x in sizes], dptr(c), float(radius), 0, None, None, None,
                                   C.byref(n))
    if code not in (0, _lib.INQB_OK) and n.value == 0:
        check(code)
    npts = n.value
    pts = np.zeros((npts, 3), np.int32)
    dist = np.zeros(npts, np.float32)
    rel = np.zeros((npts, 3), np.float32)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    check(lib.inqb_spherical_grid(dptr(lat), *[int(x) for x in sizes], dptr(c), float(radius), npts, vp(pts), vp(dist),
                                  vp(rel), C.byref(n)))
    return pts, dist, rel


# ---------------------------------------------------------------- orbital sets


class OrbitalSet:
    """states::orbital_set<real_space|fourier_space, complex> with device storage [npoint][nst]."""

    def __init__(self, basis: RealSpace, nst: int, spinor_dim: int = 1, kpoint=(0.0, 0.0, 0.0), spin_index: int = 0,
                 space: int = REAL_SPACE, precision: int = F64):
        self.basis = basis
        self.ctx = basis.ctx
        self.nst = int(nst)
        self._kpoint = np.asarray(kpoint, dtype=np.float64).copy()
        self._spin = int(spin_index)
        self.precision = precision
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.inqb_orbitals_create(self.ctx.handle, basis.handle, self.nst, spinor_dim,
                                                         dptr(self._kpoint), self._spin, space, precision, C.byref(h)))
        self.handle = h

    # --- reference-style accessors
    def set_size(self):
        return self.nst

    local_set_size = set_size

    def kpoint(self):
        return self._kpoint.copy()

    def spin_index(self):
        return self._spin

    @property
    def space(self) -> int:
        sp = C.c_int()
        self.ctx.check(self.ctx.lib.inqb_orbitals_info(self.handle, None, C.byref(sp), None, None))
        return sp.value

    @property
    def dtype(self):
        return np.complex128 if self.precision == F64 else np.complex64

    def skeleton(self, space: int | None = None) -> "OrbitalSet":
        """A new, uninitialised set with the same basis, size, k-point and spin (orbital_set::skeleton)."""
        return OrbitalSet(self.basis, self.nst, 1, self._kpoint, self._spin, self.space if space is None else space,
                          self.precision)

    def copy(self) -> "OrbitalSet":
        out = self.skeleton()
        self.ctx.check(self.ctx.lib.inqb_orbitals_copy(self.handle, out.handle))
        return out

    def assign(self, other: "OrbitalSet"):
        self.ctx.check(self.ctx.lib.inqb_orbitals_copy(other.handle, self.handle))

    def fill(self, value):
        v = complex(value)
        self.ctx.check(self.ctx.lib.inqb_orbitals_fill(self.handle, v.real, v.imag))

    def randomize_gsphere(self, seed: int, ecut: float):
        """Seeded N(0,1) Fourier coefficients inside |G|^2/2 < ecut (tags the set Fourier-space)."""
        self.ctx.check(self.ctx.lib.inqb_orbitals_randomize_gsphere(self.handle, int(seed) & (2**64 - 1), float(ecut)))
        return self

    def converted(self, precision: int) -> "OrbitalSet":
        """A copy of this set in another precision (F64 <-> F32)."""
        out = OrbitalSet(self.basis, self.nst, 1, self._kpoint, self._spin, self.space, precision)
        if precision == self.precision:
            out.assign(self)
        else:
            self.ctx.check(self.ctx.lib.inqb_orbitals_convert(self.handle, out.handle))
        return out

    def set_space(self, space: int):
        self.ctx.check(self.ctx.lib.inqb_orbitals_set_space(self.handle, space))

    def upload(self, arr):
        a = np.ascontiguousarray(np.asarray(arr).reshape(self.basis.size(), self.nst), dtype=self.dtype)
        self.ctx.check(self.ctx.lib.inqb_orbitals_upload(self.handle, a.ctypes.data_as(C.c_void_p)))
        return self

    def save(self, dirname: str) -> "OrbitalSet":
        """operations::io::save: one complex128 file per state in ``dirname`` (the reference's layout)."""
        self.ctx.check(self.ctx.lib.inqb_orbitals_save(self.handle, str(dirname).encode()))
        return self

    def load(self, dirname: str) -> "OrbitalSet":
        """operations::io::load: the states of ``dirname`` into this set."""
        self.ctx.check(self.ctx.lib.inqb_orbitals_load(self.handle, str(dirname).encode()))
        return self

    def matrix(self) -> np.ndarray:
        """Host copy [npoint][nst] (field_set::matrix())."""
        out = np.empty((self.basis.size(), self.nst), dtype=self.dtype)
        self.ctx.check(self.ctx.lib.inqb_orbitals_download(self.handle, out.ctypes.data_as(C.c_void_p)))
        return out

    def download_into(self, out: np.ndarray) -> np.ndarray:
        """Copy the set into a caller-provided contiguous host array (pinned memory copies fastest)."""
        assert out.dtype == self.dtype and out.flags.c_contiguous and out.size == self.basis.size() * self.nst
        self.ctx.check(self.ctx.lib.inqb_orbitals_download(self.handle, out.ctypes.data_as(C.c_void_p)))
        return out

    def hypercubic(self) -> np.ndarray:
        """Host copy [nx][ny][nz][nst] (field_set::hypercubic())."""
        return self.matrix().reshape(self.basis.sizes + (self.nst,))

    def device_ptr(self) -> int:
        p = C.c_void_p()
        self.ctx.check(self.ctx.lib.inqb_orbitals_device_ptr(self.handle, C.byref(p)))
        return p.value

    def nbytes(self) -> int:
        return self.basis.size() * self.nst * (16 if self.precision == F64 else 8)

    @classmethod
    def wrap(cls, basis, data_ptr: int, nst: int, kpoint=(0.0, 0.0, 0.0), spin_index: int = 0,
             space: int = REAL_SPACE, precision: int = F64, owner=None) -> "OrbitalSet":
        """A set over caller-owned device or managed storage [npoint][nst], with no copy (inqb_orbitals_wrap).
        ``owner`` (e.g. the torch tensor holding the storage) is kept alive as long as the set."""
        self = cls.__new__(cls)
        self.basis = basis
        self.ctx = basis.ctx
        self.nst = int(nst)
        self._kpoint = np.asarray(kpoint, dtype=np.float64).copy()
        self._spin = int(spin_index)
        self.precision = precision
        self._owner = owner
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.inqb_orbitals_wrap(self.ctx.handle, basis.handle, C.c_void_p(int(data_ptr)),
                                                       self.nst, 1, dptr(self._kpoint), self._spin, space, precision,
                                                       C.byref(h)))
        self.handle = h
        return self

    @classmethod
    def from_tensor(cls, basis, tensor, kpoint=(0.0, 0.0, 0.0), spin_index: int = 0, space: int = REAL_SPACE):
        """Borrow a contiguous CUDA torch tensor of complex128 or complex64 with basis.size() * nst
        elements (shape [npoint, nst] or [nx, ny, nz, nst]) as an orbital set, with no copy."""
        import torch
        if not tensor.is_cuda or not tensor.is_contiguous():
            raise ValueError("from_tensor takes a contiguous CUDA tensor")
        if tensor.dtype == torch.complex128:
            precision = F64
        elif tensor.dtype == torch.complex64:
            precision = F32
        else:
            raise ValueError("from_tensor takes complex128 or complex64")
        nst = tensor.shape[-1]
        if tensor.numel() != basis.size() * nst:
            raise ValueError(f"tensor has {tensor.numel()} elements, the basis wants {basis.size()} x {nst}")
        return cls.wrap(basis, tensor.data_ptr(), nst, kpoint, spin_index, space, precision, owner=tensor)

    @classmethod
    def from_array(cls, basis, arr, kpoint=(0.0, 0.0, 0.0), spin_index=0, space=REAL_SPACE, precision=F64):
        a = np.asarray(arr)
        nst = a.shape[-1]
        return cls(basis, nst, 1, kpoint, spin_index, space, precision).upload(a)

    def __del__(self):
        try:
            if getattr(self, "handle", None) and self.ctx.handle:
                self.ctx.lib.inqb_orbitals_destroy(self.handle)
        except Exception:
            pass


# ---------------------------------------------------------------- Hamiltonian


class KSHamiltonian:
    """hamiltonian::ks_hamiltonian with the exchange operator disabled and no relativistic projectors."""

    def __init__(self, basis: RealSpace, nspin: int = 1):
        self.basis = basis
        self.ctx = basis.ctx
        self.nspin = nspin
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.inqb_hamiltonian_create(self.ctx.handle, basis.handle, nspin, C.byref(h)))
        self.handle = h
        self._A = np.zeros(3)

    def set_option(self, key: str, value: int):
        """Kernel-option override for this Hamiltonian's applications (inqb_hamiltonian_set_option);
        a negative value (other than nl_bulk's -1) removes it."""
        self.ctx.check(self.ctx.lib.inqb_hamiltonian_set_option(self.handle, key.encode(), int(value)))

    # scalar_potential() (ks_hamiltonian.hpp:252-254): [npoint][nspin] float64
    def set_scalar_potential(self, V):
        v = np.ascontiguousarray(np.asarray(V, dtype=np.float64).reshape(self.basis.size(), self.nspin))
        self.ctx.check(self.ctx.lib.inqb_potential_set(self.handle, dptr(v)))

    def set_interaction(self, vion, hartree: bool = True, xc: str | None = "lda"):
        """The density-dependent part of the Kohn-Sham potential (self_consistency::update_hamiltonian):
        ionic potential ``vion`` [npoint], Hartree term, and ``xc`` = "lda" (Slater + PZ81) or None.
        ETRS steps then rebuild the potential from every density they form."""
        if xc not in ("lda", None):
            raise ValueError("xc is 'lda' or None")
        v = np.ascontiguousarray(np.asarray(vion, dtype=np.float64).reshape(-1))
        self._vion = v
        self.ctx.check(self.ctx.lib.inqb_hamiltonian_set_interaction(self.handle, dptr(v), int(bool(hartree)),
                                                                     1 if xc == "lda" else 0))

    def steepest_descent(self, fphi: OrbitalSet) -> OrbitalSet:
        """eigensolvers::steepest_descent with the TPA preconditioner on a Fourier-space set (in place),
        followed by orthogonalize, as one iteration of the ground-state loop calls it."""
        self.ctx.check(self.ctx.lib.inqb_steepest_descent(self.handle, fphi.handle))
        return fphi

    def clear_interaction(self):
        """Back to a fixed potential (the one in place stays until set_scalar_potential)."""
        self.ctx.check(self.ctx.lib.inqb_hamiltonian_set_interaction(self.handle, None, 0, 0))

    def update_hamiltonian(self, density) -> dict:
        """V = V_ion + V_H[n] + V_xc[n] for the density ``density`` [npoint]; returns the energies."""
        n = np.ascontiguousarray(np.asarray(density, dtype=np.float64).reshape(-1))
        e = np.zeros(4)
        self.ctx.check(self.ctx.lib.inqb_update_hamiltonian(self.handle, dptr(n), dptr(e)))
        return {"external": float(e[0]), "hartree": float(e[1]), "xc": float(e[2]), "nvxc": float(e[3])}

    @property
    def uniform_vector_potential(self):
        return self._A.copy()

    @uniform_vector_potential.setter
    def uniform_vector_potential(self, A_cov):
        self._A = np.asarray(A_cov, dtype=np.float64).copy()
        self.ctx.check(self.ctx.lib.inqb_vector_potential_set(self.handle, dptr(self._A)))

    def set_projectors(self, points, positions, matrices, coeff, npts, nlm):
        """Packed projector_all tables (see include/inqb.h inqb_projectors_set)."""
        self._moving_atoms = 0
        points = np.ascontiguousarray(points, dtype=np.int32)
        positions = np.ascontiguousarray(positions, dtype=np.float32)
        matrices = np.ascontiguousarray(matrices, dtype=np.float64)
        coeff = np.ascontiguousarray(coeff, dtype=np.float64)
        npts = np.ascontiguousarray(npts, dtype=np.int32)
        nlm = np.ascontiguousarray(nlm, dtype=np.int32)
        nproj, maxsph = points.shape[0], points.shape[1]
        maxnlm = matrices.shape[1]
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        self.ctx.check(self.ctx.lib.inqb_projectors_set(self.handle, nproj, maxsph, maxnlm, vp(points), vp(positions),
                                                        vp(matrices), vp(coeff), vp(npts), vp(nlm)))

    def update_projectors_gaussian(self, positions, radius, rc, kb, device: bool = False):
        """Synthetic KB projectors (l = 0, 1; radial exp(-r^2/rc^2)) at cartesian atom positions.
        ``device=True`` builds the spheres, values and hit lists with kernels (the host lists only the
        periodic images and their containing cubes); the tables are the same."""
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        kbv = np.ascontiguousarray(kb, dtype=np.float64).reshape(len(pos), 4, 4)
        fn = (self.ctx.lib.inqb_projectors_build_gaussian_device if device
              else self.ctx.lib.inqb_projectors_build_gaussian)
        self.ctx.check(fn(self.handle, len(pos), dptr(pos), float(radius), float(rc), dptr(kbv)))
        self._moving_atoms = len(pos)

    def move_atoms(self, positions):
        """ks_hamiltonian::update_projectors after the atoms moved (etrs.hpp:45-48): the projector
        tables rebuilt on the device for new cartesian positions, with the species parameters of the
        last Gaussian build."""
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        natoms = getattr(self, "_moving_atoms", 0)
        if natoms == 0:
            raise ValueError("no Gaussian or pseudopotential projectors were built on this Hamiltonian")
        if len(pos) != natoms:
            raise ValueError(f"{len(pos)} positions for {natoms} atoms")
        self.ctx.check(self.ctx.lib.inqb_projectors_move(self.handle, dptr(pos)))

    def projectors_info(self):
        n, m, t = C.c_int(), C.c_int(), C.c_longlong()
        self.ctx.check(self.ctx.lib.inqb_projectors_info(self.handle, C.byref(n), C.byref(m), C.byref(t)))
        return n.value, m.value, t.value

    def projector_tables(self):
        nproj, maxsph, _ = self.projectors_info()
        points = np.zeros((nproj, maxsph, 3), np.int32)
        pos = np.zeros((nproj, maxsph, 3), np.float32)
        mats = np.zeros((nproj, 4, maxsph), np.float64)
        npts = np.zeros(nproj, np.int32)
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        self.ctx.check(self.ctx.lib.inqb_projectors_get(self.handle, vp(points), vp(pos), vp(mats), vp(npts)))
        return points, pos, mats, npts

    # operator() (ks_hamiltonian.hpp:137-180)
    def __call__(self, phi: OrbitalSet) -> OrbitalSet:
        out = phi.skeleton()
        self.apply(phi, out)
        return out

    def apply(self, phi: OrbitalSet, out: OrbitalSet):
        self.ctx.check(self.ctx.lib.inqb_apply(self.handle, phi.handle, out.handle))
        return out

    def apply_host(self, host_in: np.ndarray, host_out: np.ndarray, kpoint=(0.0, 0.0, 0.0), spin_index: int = 0,
                   block_states: int = 0) -> np.ndarray:
        """H applied to a real-space set held in host memory ([npoint][nst] complex128 or complex64,
        C-contiguous); the result is written into ``host_out``.  States stream through the device in
        blocks with the copies overlapping the operator (page-locked arrays overlap, others are copied
        without overlap)."""
        if host_in.dtype != host_out.dtype or host_in.shape != host_out.shape or host_in.ndim != 2:
            raise ValueError("host_in and host_out must be [npoint][nst] arrays of one complex type")
        if host_in.dtype == np.complex128:
            prec = F64
        elif host_in.dtype == np.complex64:
            prec = F32
        else:
            raise ValueError("complex128 or complex64 arrays expected")
        if not (host_in.flags.c_contiguous and host_out.flags.c_contiguous):
            raise ValueError("host arrays must be C-contiguous")
        if host_in.shape[0] != self.basis.size():
            raise ValueError("host arrays must have one row per grid point")
        kp = np.asarray(kpoint, dtype=np.float64).copy()
        self.ctx.check(self.ctx.lib.inqb_apply_host(self.handle, int(host_in.shape[1]), kp.ctypes.data_as(_lib.DP),
                                                    int(spin_index), prec, host_in.ctypes.data, host_out.ctypes.data,
                                                    int(block_states)))
        return host_out

    def apply_host_many(self, host_ins, host_outs, kpoint=(0.0, 0.0, 0.0), spin_index: int = 0,
                        block_states: int = 0):
        """:meth:`apply_host` over several host sets of one shape in one call (inqb_apply_host_many): the
        state blocks of all sets stream through one pipeline, so consecutive sets' copies overlap."""
        host_ins, host_outs = list(host_ins), list(host_outs)
        if not host_ins or len(host_ins) != len(host_outs):
            raise ValueError("one output array per input array, at least one")
        a0 = host_ins[0]
        for a in host_ins + host_outs:
            if a.dtype != a0.dtype or a.shape != a0.shape or a.ndim != 2 or not a.flags.c_contiguous:
                raise ValueError("C-contiguous [npoint][nst] arrays of one complex type and shape expected")
        if a0.dtype == np.complex128:
            prec = F64
        elif a0.dtype == np.complex64:
            prec = F32
        else:
            raise ValueError("complex128 or complex64 arrays expected")
        if a0.shape[0] != self.basis.size():
            raise ValueError("host arrays must have one row per grid point")
        n = len(host_ins)
        ins = (C.c_void_p * n)(*[a.ctypes.data for a in host_ins])
        outs = (C.c_void_p * n)(*[a.ctypes.data for a in host_outs])
        kp = np.asarray(kpoint, dtype=np.float64).copy()
        self.ctx.check(self.ctx.lib.inqb_apply_host_many(self.handle, n, int(a0.shape[1]), kp.ctypes.data_as(_lib.DP),
                                                         int(spin_index), prec, ins, outs, int(block_states)))
        return host_outs

    def non_local(self, phi: OrbitalSet) -> OrbitalSet:
        out = phi.skeleton()
        self.ctx.check(self.ctx.lib.inqb_non_local(self.handle, phi.handle, out.handle))
        return out

    def non_local_energy(self, phi: OrbitalSet, occupations) -> float:
        occ = np.ascontiguousarray(occupations, dtype=np.float64)
        e = C.c_double()
        self.ctx.check(self.ctx.lib.inqb_non_local_energy(self.handle, phi.handle, dptr(occ), C.byref(e)))
        return e.value

    def kinetic_expectation_value(self, phi: OrbitalSet):
        out = np.zeros(phi.nst)
        self.ctx.check(self.ctx.lib.inqb_kinetic_expectation_value(self.handle, phi.handle, dptr(out)))
        return out

    def eigenvalues(self, phi: OrbitalSet):
        eig = np.zeros(phi.nst)
        res = np.zeros(phi.nst)
        self.ctx.check(self.ctx.lib.inqb_eigenvalues(self.handle, phi.handle, dptr(eig), dptr(res)))
        return eig, res

    def subspace_diagonalization(self, phi: OrbitalSet):
        """ground_state::subspace_diagonalization: rotates phi onto the subspace eigenvectors, returns eigenvalues."""
        eig = np.zeros(phi.nst)
        self.ctx.check(self.ctx.lib.inqb_subspace_diagonalization(self.handle, phi.handle, dptr(eig)))
        return eig

    def __del__(self):
        try:
            if getattr(self, "handle", None) and self.ctx.handle:
                self.ctx.lib.inqb_hamiltonian_destroy(self.handle)
        except Exception:
            pass


# ---------------------------------------------------------------- operations


def to_fourier(phi: OrbitalSet) -> OrbitalSet:
    out = phi.skeleton(FOURIER_SPACE)
    phi.ctx.check(phi.ctx.lib.inqb_to_fourier(phi.handle, out.handle))
    return out


def to_real(fphi: OrbitalSet, normalize: bool = True) -> OrbitalSet:
    out = fphi.skeleton(REAL_SPACE)
    fphi.ctx.check(fphi.ctx.lib.inqb_to_real(fphi.handle, out.handle, int(bool(normalize))))
    return out


def laplacian(fphi: OrbitalSet, factor: float = 1.0, gradcoeff=(0.0, 0.0, 0.0)) -> OrbitalSet:
    out = fphi.skeleton(FOURIER_SPACE)
    g = np.asarray(gradcoeff, dtype=np.float64)
    fphi.ctx.check(fphi.ctx.lib.inqb_laplacian(fphi.handle, out.handle, float(factor), dptr(g)))
    return out


def overlap(phi1: OrbitalSet, phi2: OrbitalSet | None = None) -> np.ndarray:
    phi2 = phi1 if phi2 is None else phi2
    out = np.zeros((phi1.nst, phi2.nst), np.complex128)
    phi1.ctx.check(phi1.ctx.lib.inqb_overlap(phi1.handle, phi2.handle, out.view(np.float64).reshape(-1).ctypes.data_as(_lib.DP)))
    return out


def overlap_diagonal(phi1: OrbitalSet, phi2: OrbitalSet | None = None) -> np.ndarray:
    phi2 = phi1 if phi2 is None else phi2
    out = np.zeros(phi1.nst, np.complex128)
    phi1.ctx.check(phi1.ctx.lib.inqb_overlap_diagonal(phi1.handle, phi2.handle,
                                                      out.view(np.float64).ctypes.data_as(_lib.DP)))
    return out


def orthogonalize(phi: OrbitalSet):
    phi.ctx.check(phi.ctx.lib.inqb_orthogonalize(phi.handle))
    return phi


def rotate(phi: OrbitalSet, R):
    r = np.ascontiguousarray(R, dtype=np.complex128)
    phi.ctx.check(phi.ctx.lib.inqb_rotate(phi.handle, r.view(np.float64).reshape(-1).ctypes.data_as(_lib.DP)))
    return phi


def rotate_to(phi: OrbitalSet, rotphi: OrbitalSet, R, alpha=1.0, beta=0.0):
    """rotphi <- alpha phi R + beta rotphi (operations::rotate with alpha and beta, rotate.hpp:83-142);
    R is [phi.nst][rotphi.nst]."""
    r = np.ascontiguousarray(R, dtype=np.complex128).reshape(phi.nst, rotphi.nst)
    a = np.array([complex(alpha).real, complex(alpha).imag])
    b = np.array([complex(beta).real, complex(beta).imag])
    phi.ctx.check(phi.ctx.lib.inqb_rotate_to(phi.handle, rotphi.handle, r.view(np.float64).reshape(-1).ctypes.data_as(_lib.DP),
                                             a.ctypes.data_as(_lib.DP), b.ctypes.data_as(_lib.DP)))
    return rotphi


def cholesky_inverse(S) -> np.ndarray:
    """U^-1 for the upper Cholesky factor of S = U^H U (matrix::cholesky, then invert_triangular), in FP64
    on the host: the matrix ``orthogonalize`` applies to a set whose overlap is S."""
    s = np.ascontiguousarray(S, dtype=np.complex128)
    n = s.shape[0]
    x = np.zeros((n, n), np.complex128)
    _lib.check(_lib.load().inqb_cholesky_inverse(n, s.view(np.float64).reshape(-1).ctypes.data_as(_lib.DP),
                                                 x.view(np.float64).reshape(-1).ctypes.data_as(_lib.DP)))
    return x


def hermitian_eigen(A):
    """(eigenvalues ascending, eigenvectors as columns) of a Hermitian matrix read from its upper
    triangle (matrix::diagonalize), in FP64 on the host: the decomposition ``subspace_diagonalization``
    uses."""
    a = np.ascontiguousarray(A, dtype=np.complex128)
    n = a.shape[0]
    w = np.zeros(n)
    v = np.zeros((n, n), np.complex128)
    _lib.check(_lib.load().inqb_hermitian_eigen(n, a.view(np.float64).reshape(-1).ctypes.data_as(_lib.DP),
                                                w.ctypes.data_as(_lib.DP),
                                                v.view(np.float64).reshape(-1).ctypes.data_as(_lib.DP)))
    return w, v


def shift(factor, chi: OrbitalSet, phi: OrbitalSet):
    f = complex(factor)
    phi.ctx.check(phi.ctx.lib.inqb_shift(f.real, f.imag, chi.handle, phi.handle))


def exponential_in_place(ham: KSHamiltonian, factor, phi: OrbitalSet, order: int = 4):
    f = complex(factor)
    ham.ctx.check(ham.ctx.lib.inqb_exponential_in_place(ham.handle, f.real, f.imag, phi.handle, order))


def exponential(ham: KSHamiltonian, factor, phi: OrbitalSet, order: int = 4) -> OrbitalSet:
    out = phi.copy()
    exponential_in_place(ham, factor, out, order)
    return out


def exponential_2_for_1(ham: KSHamiltonian, factor1, factor2, phi: OrbitalSet, order: int = 4) -> OrbitalSet:
    """Returns exp(factor1 H) phi and replaces phi by exp(factor2 H) phi (exponential.hpp:50-69)."""
    exp1 = phi.skeleton()
    f1, f2 = complex(factor1), complex(factor2)
    ham.ctx.check(ham.ctx.lib.inqb_exponential_2_for_1(ham.handle, f1.real, f1.imag, f2.real, f2.imag, phi.handle,
                                                       exp1.handle, order))
    return exp1


def _ptr_arrays(phis, occs):
    hs = (C.c_void_p * len(phis))(*[p.handle.value for p in phis])
    occ_arrays = [np.ascontiguousarray(o, dtype=np.float64) for o in occs]
    optrs = (_lib.DP * len(occs))(*[dptr(o) for o in occ_arrays])
    return hs, optrs, occ_arrays


def save_electrons(dirname: str, phis: Sequence[OrbitalSet], occupations: Sequence, spin_density) -> None:
    """systems::electrons::save (electrons.hpp:323-343): per k-point/spin set kpin<%010d>/states and
    kpin<%010d>/occupations/array, and spin_density/<component %010d> ([npoint][nspin] float64)."""
    import os
    for i, (phi, occ) in enumerate(zip(phis, occupations)):
        base = os.path.join(dirname, f"kpin{i:010d}")
        phi.save(os.path.join(base, "states"))
        o = np.ascontiguousarray(np.asarray(occ, dtype=np.float64))
        _lib.check(_lib.load().inqb_array_save(os.path.join(base, "occupations").encode(), dptr(o), o.size))
    d = np.ascontiguousarray(np.asarray(spin_density, dtype=np.float64).reshape(phis[0].basis.size(), -1))
    _lib.check(_lib.load().inqb_field_save(os.path.join(dirname, "spin_density").encode(), dptr(d), d.shape[0],
                                           d.shape[1]))


def load_electrons(dirname: str, phis: Sequence[OrbitalSet], nspin: int = 1):
    """systems::electrons::try_load (electrons.hpp:346-376): fills the sets; returns (occupations,
    spin density [npoint][nspin]).  Raises InqbError when a file is missing."""
    import os
    occs = []
    for i, phi in enumerate(phis):
        base = os.path.join(dirname, f"kpin{i:010d}")
        phi.load(os.path.join(base, "states"))
        o = np.zeros(phi.nst)
        _lib.check(_lib.load().inqb_array_load(os.path.join(base, "occupations").encode(), dptr(o), o.size))
        occs.append(o)
    d = np.zeros((phis[0].basis.size(), nspin))
    _lib.check(_lib.load().inqb_field_load(os.path.join(dirname, "spin_density").encode(), dptr(d), d.shape[0],
                                           nspin))
    return occs, d


def density(phis: Sequence[OrbitalSet], occupations: Sequence) -> np.ndarray:
    """observables::density::calculate: n = sum_sets sum_s occ_s |phi_s|^2, [npoint] float64."""
    hs, optrs, keep = _ptr_arrays(phis, occupations)
    out = np.zeros(phis[0].basis.size())
    phis[0].ctx.check(phis[0].ctx.lib.inqb_density(hs, len(phis), optrs, dptr(out)))
    return out


def dipole(basis: RealSpace, dens) -> np.ndarray:
    d = np.ascontiguousarray(dens, dtype=np.float64).reshape(-1)
    out = np.zeros(3)
    basis.ctx.check(basis.ctx.lib.inqb_dipole(basis.handle, dptr(d), dptr(out)))
    return out


class Kick:
    """perturbations::kick (kick.hpp:22-121).

    gauge 'length' multiplies the orbitals by exp(i E_cov . r) with E = -kick at the
    zero step; 'velocity' instead sets the uniform vector potential A = -kick
    (the reference's automatic choice for periodic cells)."""

    def __init__(self, cell: Cell, kick_field, gauge: str = "automatic"):
        k = np.asarray(kick_field, dtype=np.float64)
        if gauge == "automatic":
            gauge = "velocity" if cell.periodicity > 0 else "length"
        self.gauge = gauge
        self.efield = -k if gauge == "length" else np.zeros(3)
        self.vpot = -k if gauge == "velocity" else np.zeros(3)
        self.cell = cell

    def zero_step(self, phi: OrbitalSet):
        if np.any(self.efield != 0.0):
            apply_phase_kick(phi, self.efield)

    def uniform_vector_potential(self, time: float = 0.0):
        return self.vpot.copy()


def apply_phase_kick(phi: OrbitalSet, efield_cart):
    """phi *= exp(i E_cov . r) (kick::zero_step body, kick.hpp:64-69)."""
    e = np.asarray(efield_cart, dtype=np.float64)
    phi.ctx.check(phi.ctx.lib.inqb_kick(phi.handle, dptr(e)))


def etrs(ham: KSHamiltonian, phis: Sequence[OrbitalSet], occupations: Sequence, dt: float, nscf: int = 5,
         scf_threshold: float = 5e-5, want_density: bool = False, density_out=None):
    """One ETRS step (real_time/etrs.hpp:22-79); a Hamiltonian with an interaction
    (KSHamiltonian.set_interaction) is rebuilt from every density the step forms.

    Returns (density or None, electronic dipole [3], number of SCF iterations).  ``density_out``, a
    float64 CUDA tensor of basis.size() elements, receives the density on the device instead (and is
    returned in its place)."""
    hs, optrs, keep = _ptr_arrays(phis, occupations)
    dip = np.zeros(3)
    iters = C.c_int()
    if density_out is not None:
        n = phis[0].basis.size()
        if not (density_out.is_cuda and density_out.is_contiguous() and density_out.numel() == n
                and str(density_out.dtype) == "torch.float64"):
            raise ValueError("density_out must be a contiguous float64 CUDA tensor of basis.size() elements")
        dens, dens_ptr = density_out, C.cast(C.c_void_p(density_out.data_ptr()), DP)
    else:
        dens = np.zeros(phis[0].basis.size()) if want_density else None
        dens_ptr = dptr(dens) if dens is not None else None
    ham.ctx.check(ham.ctx.lib.inqb_etrs_step(ham.handle, hs, len(phis), optrs, float(dt), int(nscf), float(scf_threshold),
                                             dens_ptr, dptr(dip), C.byref(iters)))
    return dens, dip, iters.value
