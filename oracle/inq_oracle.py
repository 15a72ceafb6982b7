"""Float64 numpy restatement of the reference's H|psi> path (test infrastructure).

Array conventions follow the reference: an orbital set is ``psi[nx, ny, nz, nst]``
complex128 (``field_set::hypercubic()``, basis/field_set.hpp:232-238, state index
fastest), a potential is ``V[nx, ny, nz]`` float64 (one spin component).
Vectors carry the reference's space tags implicitly: ``*_cov`` covariant
(reciprocal-lattice components, e.g. k-points and G vectors), ``*_contra``
contravariant (fractions of the lattice vectors), otherwise cartesian.

Where bit-exact agreement with the reference matters (the sphere point selection
of spherical_grid.hpp) every float operation is written in the reference's order
with elementwise numpy arithmetic (no BLAS, no fused multiply-add).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

TWO_PI = 2.0 * math.pi

# ---------------------------------------------------------------------------
# cell / metric (systems/cell.hpp:35-215)
# ---------------------------------------------------------------------------


def _cross(a, b):
    # math/vector3.hpp:231-233
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])


def _dot3(a, b):
    # math/vector3.hpp:221-223 (left-to-right sum)
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


class Cell:
    """Lattice ``a[i]`` (rows, cartesian bohr), volume and reciprocal vectors (cell.hpp:37-53)."""

    def __init__(self, lattice, periodicity: int = 3):
        lat = np.asarray(lattice, dtype=np.float64).reshape(3, 3)
        self.lat = lat.copy()
        self.periodicity = periodicity
        self.volume = float(_dot3(lat[0], _cross(lat[1], lat[2])))
        if self.volume < 1e-10:
            raise ValueError("the lattice volume is not positive")
        pref = TWO_PI / self.volume
        self.reciprocal = np.array([pref * _cross(lat[1], lat[2]), pref * _cross(lat[2], lat[0]),
                                    pref * _cross(lat[0], lat[1])])
        # cell_metric (cell.hpp:151-160): rlat = reciprocal / 2pi
        self.rlat = self.reciprocal / TWO_PI

    @staticmethod
    def cubic(a):
        return Cell([[a, 0.0, 0.0], [0.0, a, 0.0], [0.0, 0.0, a]])

    # cell_metric conversions (cell.hpp:176-211); arrays are [..., 3]
    def contra_to_cart(self, v):
        v = np.asarray(v)
        l = self.lat
        return (l[0] * v[..., 0:1] + l[1] * v[..., 1:2]) + l[2] * v[..., 2:3]

    def cov_to_cart(self, v):
        v = np.asarray(v)
        r = self.rlat
        return (r[0] * v[..., 0:1] + r[1] * v[..., 1:2]) + r[2] * v[..., 2:3]

    def cart_to_contra(self, v):
        v = np.asarray(v)
        r = self.rlat
        return np.stack([r[k][0] * v[..., 0] + r[k][1] * v[..., 1] + r[k][2] * v[..., 2] for k in range(3)], axis=-1)

    def cart_to_cov(self, v):
        v = np.asarray(v)
        l = self.lat
        return np.stack([l[k][0] * v[..., 0] + l[k][1] * v[..., 1] + l[k][2] * v[..., 2] for k in range(3)], axis=-1)

    def cov_to_contra(self, v):
        return self.cart_to_contra(self.cov_to_cart(v))

    def norm_cov(self, v):
        c = self.cov_to_cart(v)
        return c[..., 0] * c[..., 0] + c[..., 1] * c[..., 1] + c[..., 2] * c[..., 2]

    def position_in_cell(self, pos):
        # cell.hpp:236-250
        crys = self.cart_to_contra(np.asarray(pos, dtype=np.float64))
        crys = crys - np.floor(crys)
        crys = np.where(crys >= 0.5, crys - 1.0, crys)
        return self.contra_to_cart(crys)

    def lengths(self):
        return np.sqrt(np.array([_dot3(self.lat[i], self.lat[i]) for i in range(3)]))


# ---------------------------------------------------------------------------
# grids (basis/grid.hpp, real_space.hpp, fourier_space.hpp)
# ---------------------------------------------------------------------------


def nextprod(factors, n):
    """Smallest product of ``factors`` powers that is >= n (math/nextprod.hpp)."""
    if n <= 1:
        return 1
    best = None
    # breadth search over exponents is enough for the sizes used here
    import heapq
    heap = list(factors)
    heapq.heapify(heap)
    seen = set(heap)
    while heap:
        cur = heapq.heappop(heap)
        if cur >= n:
            return cur
        for f in factors:
            c = cur * f
            if c not in seen:
                seen.add(c)
                heapq.heappush(heap, c)
    return best


def grid_dimensions(cell: Cell, spacing: float, optimize: bool = True):
    """real_space::calculate_dimensions (real_space.hpp:249-261)."""
    out = []
    for i in range(3):
        n = int(math.floor(cell.lengths()[i] / spacing + 0.5))  # C++ round() of a positive value
        if optimize:
            n = nextprod([2, 3, 5, 7], n)
        out.append(n)
    return tuple(out)


def symmetric_index(n):
    """grid::to_symmetric_range for one axis (grid.hpp:78-84)."""
    i = np.arange(n)
    return np.where(i >= (n + 1) // 2, i - n, i)


class RealSpace:
    """basis::real_space + fourier_space metric helpers on one rank."""

    def __init__(self, cell: Cell, sizes):
        self.cell = cell
        self.sizes = tuple(int(s) for s in sizes)
        self.npoints = self.sizes[0] * self.sizes[1] * self.sizes[2]
        self.conspacing = np.array([1.0 / s for s in self.sizes])
        self.rlength = cell.lengths()
        self.rspacing = self.rlength / np.array(self.sizes)

    @classmethod
    def from_spacing(cls, cell, spacing):
        return cls(cell, grid_dimensions(cell, spacing))

    def volume_element(self):
        return self.cell.volume / self.npoints  # real_space.hpp:216-218

    def fourier_volume_element(self):
        return self.cell.volume / (self.npoints * self.npoints)  # fourier_space.hpp:48-50

    def diagonal_length(self):
        r = self.rlength
        return math.sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2])

    def rvector_contra(self):
        """[nx,ny,nz,3] contravariant point positions, symmetric range (real_space.hpp:127-135)."""
        sx, sy, sz = (symmetric_index(n) for n in self.sizes)
        c = self.conspacing
        X, Y, Z = np.meshgrid(sx * c[0], sy * c[1], sz * c[2], indexing="ij")
        return np.stack([X, Y, Z], axis=-1)

    def rvector_cartesian(self):
        return self.cell.contra_to_cart(self.rvector_contra())

    def r2(self):
        r = self.rvector_cartesian()
        return r[..., 0] * r[..., 0] + r[..., 1] * r[..., 1] + r[..., 2] * r[..., 2]

    def gvector_cov(self):
        """[nx,ny,nz,3] covariant G = 2pi * symmetric index (fourier_space.hpp:77-85, serial order)."""
        sx, sy, sz = (symmetric_index(n) for n in self.sizes)
        X, Y, Z = np.meshgrid(sx * TWO_PI, sy * TWO_PI, sz * TWO_PI, indexing="ij")
        return np.stack([X, Y, Z], axis=-1)

    def g2(self):
        return self.cell.norm_cov(self.gvector_cov())

    def outside_sphere(self):
        """fourier_space point_operator::outside_sphere (fourier_space.hpp:93-99)."""
        sx, sy, sz = (symmetric_index(n) / n for n in self.sizes)
        X, Y, Z = np.meshgrid(sx, sy, sz, indexing="ij")
        return X * X + Y * Y + Z * Z > 0.25


# ---------------------------------------------------------------------------
# spherical grid (basis/spherical_grid.hpp:59-160, containing_cube.hpp:20-45,
# ionic/periodic_replicas.hpp:22-60)
# ---------------------------------------------------------------------------


def periodic_replicas(cell: Cell, position, range_):
    position = cell.position_in_cell(np.asarray(position, dtype=np.float64))
    reps = [position]
    nmax = [0, 0, 0]
    for d in range(cell.periodicity):
        nmax[d] = 1 + int(_lround(range_ / math.sqrt(_dot3(cell.lat[d], cell.lat[d]))))
    for ix in range(-nmax[0], nmax[0] + 1):
        for iy in range(-nmax[1], nmax[1] + 1):
            for iz in range(-nmax[2], nmax[2] + 1):
                if ix == 0 and iy == 0 and iz == 0:
                    continue
                rep = ((position + ix * cell.lat[0]) + iy * cell.lat[1]) + iz * cell.lat[2]
                reps.append(rep)
    return reps


def _lround(x):
    # C lround: half away from zero
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)


def containing_cube(rs: RealSpace, pos, radius):
    lo = [0, 0, 0]
    hi = [0, 0, 0]
    for d in range(3):
        rec = rs.cell.reciprocal[d]
        lrec = math.sqrt(_dot3(rec, rec))
        sc = radius / lrec
        lointer = pos - sc * rec
        hiinter = pos + sc * rec
        r = rs.cell.rlat[d]
        dlo = r[0] * lointer[0] + r[1] * lointer[1] + r[2] * lointer[2]
        dhi = r[0] * hiinter[0] + r[1] * hiinter[1] + r[2] * hiinter[2]
        n = rs.sizes[d]
        lo[d] = _lround(math.floor(dlo / rs.conspacing[d]))
        hi[d] = _lround(math.ceil(dhi / rs.conspacing[d])) + 1
        b, e = -(n // 2), n // 2 + n % 2
        lo[d] = min(max(lo[d], b), e)
        hi[d] = min(max(hi[d], b), e)
    return lo, hi


@dataclass
class Sphere:
    points: np.ndarray      # [npts, 3] int32 grid indices in [0, n)
    distance: np.ndarray    # [npts] float32
    relpos: np.ndarray      # [npts, 3] float32 contravariant offset from the (replica) centre

    @property
    def size(self):
        return len(self.points)


def spherical_grid(rs: RealSpace, center, radius) -> Sphere:
    """Points of ``rs`` within ``radius`` of ``center`` or any periodic image.

    Order, float32 storage of distance / relative position and the selection test
    ``|r - R|^2 > radius^2`` follow spherical_grid.hpp:59-160 exactly (replica loop,
    then x-major / z-fastest cube scan, stable compaction).
    """
    reps = periodic_replicas(rs.cell, center, rs.diagonal_length())
    pts, dist, rel = [], [], []
    lat = rs.cell.lat
    for re in reps:
        lo, hi = containing_cube(rs, re, radius)
        dims = [hi[d] - lo[d] for d in range(3)]
        if dims[0] * dims[1] * dims[2] <= 0:
            continue
        ii = [np.arange(lo[d], hi[d]) for d in range(3)]
        I = np.meshgrid(*ii, indexing="ij")
        gidx = []
        contra = []
        for d in range(3):
            n = rs.sizes[d]
            g = np.where(I[d] < 0, I[d] + n, I[d])          # from_symmetric_range
            s = np.where(g >= (n + 1) // 2, g - n, g)       # to_symmetric_range
            gidx.append(g)
            contra.append(s * rs.conspacing[d])
        # to_cartesian(contra): lat0*v0 + lat1*v1 + lat2*v2, componentwise
        rp = [(lat[0][j] * contra[0] + lat[1][j] * contra[1]) + lat[2][j] * contra[2] for j in range(3)]
        df = [rp[j] - re[j] for j in range(3)]
        n2 = df[0] * df[0] + df[1] * df[1] + df[2] * df[2]
        keep = ~(n2 > radius * radius)
        if not keep.any():
            continue
        r = rs.cell.rlat
        cpos = [r[k][0] * df[0] + r[k][1] * df[1] + r[k][2] * df[2] for k in range(3)]
        pts.append(np.stack([gidx[0][keep], gidx[1][keep], gidx[2][keep]], axis=-1).reshape(-1, 3))
        dist.append(np.sqrt(n2[keep]).astype(np.float32).reshape(-1))
        rel.append(np.stack([cpos[0][keep], cpos[1][keep], cpos[2][keep]], axis=-1).astype(np.float32).reshape(-1, 3))
    if not pts:
        return Sphere(np.zeros((0, 3), np.int32), np.zeros(0, np.float32), np.zeros((0, 3), np.float32))
    return Sphere(np.concatenate(pts).astype(np.int32), np.concatenate(dist), np.concatenate(rel))


# ---------------------------------------------------------------------------
# projectors (hamiltonian/projector.hpp:38-113, projector_all.hpp:40-109)
# ---------------------------------------------------------------------------

Y00 = 0.5 / math.sqrt(math.pi)
Y1 = math.sqrt(3.0 / (4.0 * math.pi))


def real_ylm(l, m, cart):
    """Real spherical harmonics used by the synthetic projectors.

    Convention (the reference's sharmonic::cartesian_real is an absent submodule):
    Y_00 = 1/(2 sqrt(pi)); Y_1,{-1,0,1} = sqrt(3/4pi) * {y, z, x}/r; Y_1m = 0 at r = 0.
    """
    cart = np.asarray(cart, dtype=np.float64)
    if l == 0:
        return np.full(cart.shape[:-1], Y00)
    r = np.sqrt(cart[..., 0] * cart[..., 0] + cart[..., 1] * cart[..., 1] + cart[..., 2] * cart[..., 2])
    comp = {-1: 1, 0: 2, 1: 0}[m]
    with np.errstate(invalid="ignore", divide="ignore"):
        v = np.where(r > 0.0, Y1 * cart[..., comp] / np.where(r > 0.0, r, 1.0), 0.0)
    return v


def gaussian_radial(distance_f32, rc):
    d = np.asarray(distance_f32, dtype=np.float64)
    return np.exp(-(d * d) / (rc * rc))


def kb_m_matching(kb_l, ls):
    """4x4 (nlm x nlm) KB matrix from per-l-projector coefficients (projector.hpp:41-93)."""
    proj_m, proj_i = [], []
    for il, l in enumerate(ls):
        for mm in range(2 * l + 1):
            proj_m.append(mm)
            proj_i.append(il)
    n = len(proj_m)
    out = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            out[i, j] = 0.0 if proj_m[i] != proj_m[j] else kb_l[proj_i[i], proj_i[j]]
    return out


@dataclass
class Projector:
    sphere: Sphere
    matrix: np.ndarray   # [nlm, npts] float64
    kb: np.ndarray       # [nlm, nlm]


def build_projector(rs: RealSpace, center, radius, rc, kb_lm, ls=(0, 1)):
    sph = spherical_grid(rs, center, radius)
    nlm = sum(2 * l + 1 for l in ls)
    mat = np.zeros((nlm, sph.size))
    if sph.size:
        cart = rs.cell.contra_to_cart(sph.relpos.astype(np.float64))
        rad = gaussian_radial(sph.distance, rc)
        ilm = 0
        for l in ls:
            for mm in range(2 * l + 1):
                mat[ilm] = rad * real_ylm(l, mm - l, cart)
                ilm += 1
    return Projector(sph, mat, np.asarray(kb_lm, dtype=np.float64))


@dataclass
class ProjectorAll:
    """Padded projector tensors (projector_all.hpp:40-89)."""
    points: np.ndarray    # [nproj, maxsph, 3] int32, -1 padded
    positions: np.ndarray  # [nproj, maxsph, 3] float32
    matrices: np.ndarray  # [nproj, nlm, maxsph]
    coeff: np.ndarray     # [nproj, nlm, nlm]
    npts: np.ndarray      # [nproj]
    nlm: np.ndarray       # [nproj]

    @property
    def nproj(self):
        return len(self.npts)

    @classmethod
    def pack(cls, projs):
        nproj = len(projs)
        maxsph = max([p.sphere.size for p in projs] + [0])
        maxnlm = max([p.matrix.shape[0] for p in projs] + [0])
        points = np.full((nproj, maxsph, 3), -1, np.int32)
        pos = np.zeros((nproj, maxsph, 3), np.float32)
        mats = np.zeros((nproj, maxnlm, maxsph))
        coeff = np.zeros((nproj, maxnlm, maxnlm))
        for i, p in enumerate(projs):
            n = p.sphere.size
            nl = p.matrix.shape[0]
            points[i, :n] = p.sphere.points
            pos[i, :n] = p.sphere.relpos
            mats[i, :nl, :n] = p.matrix
            coeff[i, :nl, :nl] = p.kb
        return cls(points, pos, mats, coeff, np.array([p.sphere.size for p in projs], np.int32),
                   np.array([p.matrix.shape[0] for p in projs], np.int32))


# ---------------------------------------------------------------------------
# operator pieces
# ---------------------------------------------------------------------------


_FFT_WORKERS = None


def set_fft_workers(n):
    """Use scipy's pocketfft with ``n`` threads for the transforms (CPU baseline timing)."""
    global _FFT_WORKERS
    _FFT_WORKERS = n


def to_fourier(psi):
    """transform::to_fourier serial path (transform.hpp:52-80): unnormalised forward DFT (e^{-iGr})."""
    if _FFT_WORKERS:
        import scipy.fft
        return scipy.fft.fftn(psi, axes=(0, 1, 2), workers=_FFT_WORKERS)
    return np.fft.fftn(psi, axes=(0, 1, 2))


def to_real(fpsi, normalize=True):
    """transform::to_real serial path (transform.hpp:113-182): backward DFT, times 1/N when normalising."""
    if _FFT_WORKERS:
        import scipy.fft
        out = scipy.fft.ifftn(fpsi, axes=(0, 1, 2), workers=_FFT_WORKERS)
    else:
        out = np.fft.ifftn(fpsi, axes=(0, 1, 2))
    if not normalize:
        out = out * (fpsi.shape[0] * fpsi.shape[1] * fpsi.shape[2])
    return out


def laplacian_factor(rs: RealSpace, factor=1.0, gradcoeff_contra=(0.0, 0.0, 0.0)):
    """factor*(-|G|^2 + gradcoeff . G) per Fourier point (laplacian.hpp:24-81)."""
    G = rs.gvector_cov()
    gc = np.asarray(gradcoeff_contra, dtype=np.float64)
    return factor * (-rs.g2() + (gc[0] * G[..., 0] + gc[1] * G[..., 1] + gc[2] * G[..., 2]))


def laplacian(rs, fpsi, factor=1.0, gradcoeff_contra=(0.0, 0.0, 0.0)):
    return laplacian_factor(rs, factor, gradcoeff_contra)[..., None] * fpsi


def laplacian_expectation_value(rs, fpsi, factor=1.0, gradcoeff_contra=(0.0, 0.0, 0.0)):
    """laplacian.hpp:85-117: dV_fs * sum conj(f) lapl f, with the -|k+A|^2/4-style constant k2."""
    gc = np.asarray(gradcoeff_contra, dtype=np.float64)
    gcart = rs.cell.contra_to_cart(gc)
    k2 = -0.25 * float(_dot3(gcart, gcart))
    G = rs.gvector_cov()
    fac = factor * rs.fourier_volume_element()
    lapl = fac * (-rs.g2() + (gc[0] * G[..., 0] + gc[1] * G[..., 1] + gc[2] * G[..., 2]) + k2)
    return np.real(np.sum(np.conj(fpsi) * lapl[..., None] * fpsi, axis=(0, 1, 2)))


def bloch_phase(pa: ProjectorAll, kpoint_cov, sign=+1.0):
    """polar(1, +-k . pos) per sphere point (projector_all.hpp:124,283); pos is the float32 table."""
    k = np.asarray(kpoint_cov, dtype=np.float64)
    pos = pa.positions.astype(np.float64)
    arg = k[0] * pos[..., 0] + k[1] * pos[..., 1] + k[2] * pos[..., 2]
    return np.exp(1j * sign * arg)


def calculate_projections(rs, pa: ProjectorAll, psi, kpoint_cov):
    """gather + gemm_1 (projector_all.hpp:113-189): proj[p,l,s] = dV sum_i M[p,l,i] e^{ik.r_i} psi[r_i,s]."""
    nst = psi.shape[-1]
    maxsph = pa.points.shape[1]
    out = np.zeros((pa.nproj, pa.matrices.shape[1], nst), complex)
    if maxsph == 0:
        return out
    ph = bloch_phase(pa, kpoint_cov, +1.0)
    for p in range(pa.nproj):
        n = pa.npts[p]
        pts = pa.points[p, :n]
        sph = ph[p, :n, None] * psi[pts[:, 0], pts[:, 1], pts[:, 2], :]
        out[p] = rs.volume_element() * (pa.matrices[p][:, :n] @ sph)
    return out


def multiply_by_coefficients(pa: ProjectorAll, proj):
    """projector_all.hpp:193-211: proj'[p,l,s] = sum_j coe[p,l,j] proj[p,j,s]."""
    return np.einsum("plj,pjs->pls", pa.coeff, proj)


def project(rs, pa, psi, kpoint_cov):
    """projector_all::project (projector_all.hpp:215-272): returns sphere_phi_all[p, i, s]."""
    proj = multiply_by_coefficients(pa, calculate_projections(rs, pa, psi, kpoint_cov))
    return np.einsum("pli,pls->pis", pa.matrices, proj)


def apply_projectors(pa, sphere_v, hpsi, kpoint_cov):
    """projector_all::apply (projector_all.hpp:276-288): hpsi[r_i] += e^{-ik.r_i} sphere_v[p,i]."""
    ph = bloch_phase(pa, kpoint_cov, -1.0)
    for p in range(pa.nproj):
        n = pa.npts[p]
        pts = pa.points[p, :n]
        np.add.at(hpsi, (pts[:, 0], pts[:, 1], pts[:, 2]), ph[p, :n, None] * sphere_v[p, :n])
    return hpsi


def non_local_energy(rs, pa, psi, kpoint_cov, occupations):
    """projector_all::energy (projector_all.hpp:306-327)."""
    proj = calculate_projections(rs, pa, psi, kpoint_cov)
    dproj = multiply_by_coefficients(pa, proj)
    occ = np.asarray(occupations, dtype=np.float64)
    return float(np.sum(occ[None, None, :] * np.real(np.conj(proj) * dproj)))


@dataclass
class Hamiltonian:
    """ks_hamiltonian<complex|double> with exchange disabled and no relativistic projectors."""
    rs: RealSpace
    V: np.ndarray                      # [nx,ny,nz] scalar potential of this spin index
    pa: ProjectorAll | None = None
    A_cov: np.ndarray = field(default_factory=lambda: np.zeros(3))

    def kA(self, kpoint_cov):
        return np.asarray(kpoint_cov, dtype=np.float64) + self.A_cov

    def _kinetic_factor(self, kA):
        # the per-point factor -0.5*(-|G|^2 + gc.G) depends only on k + A: keep the last one
        key = tuple(float(v) for v in kA)
        if getattr(self, "_kin_key", None) != key:
            gradcoeff = -2.0 * self.rs.cell.cov_to_contra(kA)
            self._kin = laplacian_factor(self.rs, -0.5, gradcoeff)[..., None]
            self._kin_key = key
        return self._kin

    def apply_real(self, psi, kpoint_cov=(0.0, 0.0, 0.0)):
        """ks_hamiltonian::operator()(orbital_set<real_space>) (ks_hamiltonian.hpp:137-156)."""
        kA = self.kA(kpoint_cov)
        sphere = project(self.rs, self.pa, psi, kA) if self.pa is not None and self.pa.nproj else None
        fpsi = to_fourier(psi)
        hf = self._kinetic_factor(kA) * fpsi
        hpsi = to_real(hf)
        shift = 0.5 * float(self.rs.cell.norm_cov(kA))
        hpsi = hpsi + (self.V[..., None] + shift) * psi
        if sphere is not None:
            apply_projectors(self.pa, sphere, hpsi, kA)
        return hpsi

    def apply_fourier(self, fpsi, kpoint_cov=(0.0, 0.0, 0.0)):
        """ks_hamiltonian::operator()(orbital_set<fourier_space>) (ks_hamiltonian.hpp:160-180)."""
        kA = self.kA(kpoint_cov)
        psi = to_real(fpsi)
        sphere = project(self.rs, self.pa, psi, kA) if self.pa is not None and self.pa.nproj else None
        shift = 0.5 * float(self.rs.cell.norm_cov(kA))
        hpsi = (self.V[..., None] + shift) * psi
        if sphere is not None:
            apply_projectors(self.pa, sphere, hpsi, kA)
        hf = to_fourier(hpsi)
        gradcoeff = -2.0 * self.rs.cell.cov_to_contra(kA)
        return hf + laplacian(self.rs, fpsi, -0.5, gradcoeff)

    def non_local(self, psi, kpoint_cov=(0.0, 0.0, 0.0)):
        kA = self.kA(kpoint_cov)
        out = np.zeros_like(psi)
        if self.pa is not None and self.pa.nproj:
            apply_projectors(self.pa, project(self.rs, self.pa, psi, kA), out, kA)
        return out

    def non_local_energy(self, psi, occupations, kpoint_cov=(0.0, 0.0, 0.0)):
        if self.pa is None or not self.pa.nproj:
            return 0.0
        return non_local_energy(self.rs, self.pa, psi, self.kA(kpoint_cov), occupations)

    def kinetic_expectation_value(self, psi, kpoint_cov=(0.0, 0.0, 0.0)):
        kA = self.kA(kpoint_cov)
        return laplacian_expectation_value(self.rs, to_fourier(psi), -0.5, -2.0 * self.rs.cell.cov_to_contra(kA))


# ---------------------------------------------------------------------------
# linear algebra on orbital sets (operations/overlap*.hpp, orthogonalize.hpp)
# ---------------------------------------------------------------------------


def overlap(rs, phi1, phi2=None):
    """S[i,j] = dV sum_r conj(phi1[r,i]) phi2[r,j] (overlap.hpp:26-41)."""
    if phi2 is None:
        phi2 = phi1
    a = phi1.reshape(-1, phi1.shape[-1])
    b = phi2.reshape(-1, phi2.shape[-1])
    return rs.volume_element() * (a.conj().T @ b)


def overlap_diagonal(rs, phi1, phi2=None):
    """d[i] = dV sum_r conj(phi1[r,i]) phi2[r,i] (overlap_diagonal.hpp:25-55)."""
    if phi2 is None:
        phi2 = phi1
    return rs.volume_element() * np.sum(np.conj(phi1) * phi2, axis=(0, 1, 2))


def orthogonalize(rs, phi):
    """orthogonalize.hpp:25-31: S = U^H U (upper Cholesky), phi <- phi U^{-1}."""
    S = overlap(rs, phi)
    L = np.linalg.cholesky(S)            # S = L L^H, U = L^H
    U = L.conj().T
    Uinv = np.linalg.inv(U)
    shp = phi.shape
    return (phi.reshape(-1, shp[-1]) @ Uinv).reshape(shp)


def subspace_diagonalization(ham: Hamiltonian, phi, kpoint_cov=(0.0, 0.0, 0.0)):
    """subspace_diagonalization.hpp:21-29: H_sub = <phi|H phi>, Hermitian eigenproblem (upper triangle),
    phi rotated onto the eigenvectors; eigenvalues ascending."""
    Hs = overlap(ham.rs, phi, ham.apply_real(phi, kpoint_cov))
    w, U = np.linalg.eigh(Hs, UPLO="U")
    shp = phi.shape
    return w, (phi.reshape(-1, shp[-1]) @ U).reshape(shp)


def eigenvalues(ham: Hamiltonian, phi, kpoint_cov=(0.0, 0.0, 0.0)):
    """energy::calculate eigenvalue part (energy.hpp:83-89): Re<phi|H phi>/<phi|phi>, residual norms."""
    hphi = ham.apply_real(phi, kpoint_cov)
    norms = np.real(overlap_diagonal(ham.rs, phi))
    eig = np.real(overlap_diagonal(ham.rs, phi, hphi)) / norms
    res = hphi - eig[None, None, None, :] * phi
    return eig, np.real(overlap_diagonal(ham.rs, res))


# ---------------------------------------------------------------------------
# real-time pieces (operations/exponential.hpp, real_time/etrs.hpp, observables)
# ---------------------------------------------------------------------------


def exponential_in_place(apply, factor, phi, order=4):
    """exponential.hpp:21-34: phi += sum_{n=1..order} factor^n/n! H^n phi."""
    hn = apply(phi)
    coeff = 1.0 + 0.0j
    phi = phi.copy()
    for it in range(1, order + 1):
        if it > 1:
            hn = apply(hn)
        coeff = coeff * factor / it
        phi += coeff * hn
    return phi


def exponential_2_for_1(apply, factor1, factor2, phi, order=4):
    """exponential.hpp:50-69: returns (exp(factor1 H) phi, exp(factor2 H) phi) from one set of H^n phi."""
    exp1 = phi.copy()
    exp2 = phi.copy()
    hn = apply(phi)
    c1 = 1.0 + 0.0j
    c2 = 1.0 + 0.0j
    for it in range(1, order + 1):
        if it > 1:
            hn = apply(hn)
        c1 = c1 * factor1 / it
        c2 = c2 * factor2 / it
        exp1 += c1 * hn
        exp2 += c2 * hn
    return exp1, exp2


def density(phi_list, occ_list, nspin=1, spin_index=None):
    """density::calculate (density.hpp:24-101), non-spinor: n = sum_s f_s |phi_s|^2."""
    n = None
    for phi, occ in zip(phi_list, occ_list):
        d = np.sum(np.asarray(occ)[None, None, None, :] * (phi.real * phi.real + phi.imag * phi.imag), axis=-1)
        n = d if n is None else n + d
    return n


def integral_sum_absdiff(rs, a, b):
    """operations::integral_sum_absdiff: dV * sum |a - b| over all points and components."""
    return rs.volume_element() * float(np.sum(np.abs(a - b)))


def dipole_electronic(rs, dens):
    """observables::dipole(density) (dipole.hpp:24-40): dV * sum r n(r), r in the symmetric range."""
    r = rs.rvector_cartesian()
    return rs.volume_element() * np.sum(r * dens[..., None], axis=(0, 1, 2))


def kick_phase(rs, phi, efield_cart):
    """kick::zero_step (kick.hpp:58-70): phi *= exp(i E_cov . r_contra)."""
    cov = rs.cell.cart_to_cov(np.asarray(efield_cart, dtype=np.float64))
    rc = rs.rvector_contra()
    arg = cov[0] * rc[..., 0] + cov[1] * rc[..., 1] + cov[2] * rc[..., 2]
    return phi * np.exp(1j * arg)[..., None]


def etrs_step(ham: Hamiltonian, phis, occs, dt, kpoints=None, nscf=5, scf_threshold=5e-5,
              update_hamiltonian=None):
    """One ETRS step (etrs.hpp:22-79) for a fixed (non-interacting) Hamiltonian.

    ``update_hamiltonian(density)`` is the self-consistency hook; with ``None`` the
    Hamiltonian is kept (static ions, no Hartree/XC), which is what the synthetic
    configurations use.  Returns (new phis, density, number of SCF iterations).
    """
    if kpoints is None:
        kpoints = [(0.0, 0.0, 0.0)] * len(phis)
    save = []
    predicted = []
    for phi, kp in zip(phis, kpoints):
        half, full = exponential_2_for_1(lambda x, kp=kp: ham.apply_real(x, kp), complex(0.0, -dt / 2.0),
                                         complex(0.0, -dt), phi)
        save.append(half)
        predicted.append(full)
    dens = density(predicted, occs)
    if update_hamiltonian is not None:
        update_hamiltonian(dens)
    cur = [s.copy() for s in save]
    iters = 0
    for iscf in range(nscf):
        cur = []
        for s, kp in zip(save, kpoints):
            cur.append(exponential_in_place(lambda x, kp=kp: ham.apply_real(x, kp), complex(0.0, -dt / 2.0), s))
        old = dens
        dens = density(cur, occs)
        delta = integral_sum_absdiff(ham.rs, old, dens)
        done = delta < scf_threshold or iscf == nscf - 1
        if update_hamiltonian is not None:
            update_hamiltonian(dens)
        iters = iscf + 1
        if done:
            break
    return cur, dens, iters


# ---------------------------------------------------------------------------
# interacting Hamiltonian update (solvers/poisson.hpp, hamiltonian/xc_term.hpp,
# hamiltonian/self_consistency.hpp)
# ---------------------------------------------------------------------------


def poisson_solve(rs: RealSpace, density):
    """solvers::poisson::solve for a periodic cell (poisson.hpp:98-104 with poisson_apply_kernel
    :72-87 and poisson_kernel_3d :29-35): V(G) = 4 pi n(G) / |G|^2 (cartesian |G|^2), the G with
    |G|^2 < 1e-6 set to the zero term 0, unnormalised backward transform.  A real density gives a
    real potential (the real part, poisson.hpp:207-212)."""
    real_in = np.isrealobj(density)
    d = np.asarray(density, dtype=np.complex128)[..., None]
    fd = to_fourier(d)
    g2 = rs.g2()
    scal = (-4.0 * math.pi) / rs.npoints
    kern = np.where(g2 < 1e-6, 0.0, -1.0 / np.where(g2 < 1e-6, 1.0, g2))
    fd = fd * (scal * kern)[..., None]
    v = to_real(fd, normalize=False)[..., 0]
    return v.real if real_in else v


LDA_X_FACTOR = -0.75 * (3.0 / math.pi) ** (1.0 / 3.0)   # eps_x = LDA_X_FACTOR n^(1/3)
PZ_GAMMA, PZ_BETA1, PZ_BETA2 = -0.1423, 1.0529, 0.3334  # Perdew-Zunger 1981, rs >= 1
PZ_A, PZ_B, PZ_C, PZ_D = 0.0311, -0.048, 0.0020, -0.0116  # rs < 1
DENS_THRESHOLD = 1e-15


def lda_x(n):
    """Slater exchange of an unpolarised density (libxc XC_LDA_X): energy per particle and potential."""
    n = np.asarray(n, dtype=np.float64)
    ok = n > DENS_THRESHOLD
    nc = np.where(ok, n, 1.0)
    eps = np.where(ok, LDA_X_FACTOR * np.cbrt(nc), 0.0)
    return eps, 4.0 / 3.0 * eps


def lda_c_pz(n):
    """Perdew-Zunger 1981 correlation of an unpolarised density (libxc XC_LDA_C_PZ, the published
    parametrisation): energy per particle and potential v = eps - rs/3 deps/drs."""
    n = np.asarray(n, dtype=np.float64)
    ok = n > DENS_THRESHOLD
    rs = np.cbrt(3.0 / (4.0 * math.pi * np.where(ok, n, 1.0)))
    sq = np.sqrt(rs)
    den = 1.0 + PZ_BETA1 * sq + PZ_BETA2 * rs
    eps_hi = PZ_GAMMA / den
    v_hi = eps_hi * (1.0 + 7.0 / 6.0 * PZ_BETA1 * sq + 4.0 / 3.0 * PZ_BETA2 * rs) / den
    lr = np.log(rs)
    eps_lo = PZ_A * lr + PZ_B + PZ_C * rs * lr + PZ_D * rs
    v_lo = PZ_A * lr + (PZ_B - PZ_A / 3.0) + 2.0 / 3.0 * PZ_C * rs * lr + (2.0 * PZ_D - PZ_C) / 3.0 * rs
    eps = np.where(rs >= 1.0, eps_hi, eps_lo)
    v = np.where(rs >= 1.0, v_hi, v_lo)
    return np.where(ok, eps, 0.0), np.where(ok, v, 0.0)


def xc_lda(rs: RealSpace, n):
    """xc_term with the LDA (options::theory::lda, theory.hpp:48-54: Slater exchange + PZ
    correlation), unpolarised: returns (v_xc, E_xc = int n eps_xc, int n v_xc) (xc_term.hpp:186-236)."""
    ex, vx = lda_x(n)
    ec, vc = lda_c_pz(n)
    v = vx + vc
    dv = rs.volume_element()
    return v, dv * float(np.sum(n * (ex + ec))), dv * float(np.sum(n * v))


def update_hamiltonian(ham: Hamiltonian, vion, n, hartree=True, xc=True):
    """self_consistency::update_hamiltonian (self_consistency.hpp:88-170), unpolarised, static ions, no
    external fields: V = V_ion + V_H[n] + V_xc[n]; returns the energies (external, Hartree, xc, nvxc)."""
    dv = ham.rs.volume_element()
    v = np.array(vion, dtype=np.float64, copy=True)
    energies = {"external": dv * float(np.sum(n * vion)), "hartree": 0.0, "xc": 0.0, "nvxc": 0.0}
    if hartree:
        vh = poisson_solve(ham.rs, n)
        energies["hartree"] = 0.5 * dv * float(np.sum(n * vh))
        v = v + vh
    if xc:
        vxc, exc, nvxc = xc_lda(ham.rs, n)
        energies["xc"], energies["nvxc"] = exc, nvxc
        v = v + vxc
    ham.V = v
    return energies


# ---------------------------------------------------------------------------
# Fourier-space eigensolver (eigensolvers/steepest_descent.hpp, operations/preconditioner.hpp)
# ---------------------------------------------------------------------------


def tpa_k(x):
    """Teter-Payne-Allan preconditioner function (preconditioner.hpp:24-30)."""
    num = ((8.0 * x + 12.0) * x + 18.0) * x + 27.0
    den = (((16.0 * x + 8.0) * x + 12.0) * x + 18.0) * x + 27.0
    return num / den


def precondition(rs: RealSpace, fphi):
    """preconditioner::operator()(orbital_set<fourier_space>) (preconditioner.hpp:32-46): each state times
    K(0.5 |G|^2 / T_s), T_s = Re <-0.5 lapl phi_s | phi_s> / <phi_s | phi_s>."""
    lap = laplacian(rs, fphi, -0.5)
    kin = np.real(np.sum(np.conj(lap) * fphi, axis=(0, 1, 2)) / np.sum(np.conj(fphi) * fphi, axis=(0, 1, 2)))
    lapl = 0.5 * rs.g2()
    return fphi * tpa_k(lapl[..., None] / kin[None, None, None, :])


def overlap_diagonal_fs(rs: RealSpace, a, b=None):
    """overlap_diagonal of Fourier-space sets: the Fourier volume element Omega / N^2."""
    if b is None:
        b = a
    return rs.fourier_volume_element() * np.sum(np.conj(a) * b, axis=(0, 1, 2))


def orthogonalize_fs(rs: RealSpace, fphi):
    """orthogonalize.hpp:25-31 on a Fourier-space set (overlap with Omega / N^2)."""
    S = rs.fourier_volume_element() * np.einsum("xyzi,xyzj->ij", np.conj(fphi), fphi)
    U = np.linalg.cholesky(S).conj().T
    shp = fphi.shape
    return (fphi.reshape(-1, shp[-1]) @ np.linalg.inv(U)).reshape(shp)


def steepest_descent(ham: Hamiltonian, fphi, kpoint_cov=(0.0, 0.0, 0.0), num_steps=5):
    """eigensolvers::steepest_descent (steepest_descent.hpp:23-86) with the TPA preconditioner on a
    Fourier-space set; returns the new set (orthonormalised)."""
    rs = ham.rs
    phi = fphi.copy()
    hphi = ham.apply_fourier(phi, kpoint_cov)
    for istep in range(num_steps):
        res = hphi.copy()
        ev = overlap_diagonal_fs(rs, res, phi)
        norm = overlap_diagonal_fs(rs, phi)
        evnorm = ev / np.real(norm)
        res = res - evnorm[None, None, None, :] * phi            # shift(-1, evnorm, phi, residual)
        res = precondition(rs, res)
        hres = ham.apply_fourier(res, kpoint_cov)
        m0 = overlap_diagonal_fs(rs, res, res)
        m1 = overlap_diagonal_fs(rs, phi, res)
        m2 = overlap_diagonal_fs(rs, res, hres)
        m3 = overlap_diagonal_fs(rs, phi, hres)
        m4, m5 = ev, norm
        ca = np.real(m0 * m3 - m2 * m1)
        cb = np.real(m5 * m2 - m4 * m0)
        cc = np.real(m4 * m1 - m3 * m5)
        den = cb + np.sqrt(cb * cb - 4.0 * ca * cc)
        lam = np.where(np.abs(den) < 1e-15, 0.0, 2.0 * cc / np.where(np.abs(den) < 1e-15, 1.0, den))
        phi = phi + lam[None, None, None, :] * res
        if istep != num_steps - 1:
            hphi = hphi + lam[None, None, None, :] * hres
    return orthogonalize_fs(rs, phi)
