"""Norm-conserving pseudopotentials from UPF files and the nonlocal projectors built from them.

This is the part of the pseudopotential reader (the reference reads pseudopotentials through its
pseudopod submodule, hamiltonian/atomic_potential.hpp) that the H|psi> path needs: the radial
mesh, the local potential and the Kleinman-Bylander projectors beta_i(r) with their coefficients
D_ij.  Both UPF layouts are read: version 2 (XML elements with attributes) and version 1 (the older
text blocks).  UPF files hold energies in Rydberg: the local potential and D_ij are converted to
Hartree, so the KB coefficients are D_ij / 2 (the values the reference's projector test expects for
its N.upf and N_non_diagonal.upf files, projector.hpp:160-240).  PP_BETA holds r * beta(r); the
projector functions here are beta(r) = (r beta)(r) / r.

``projector_tables`` builds, for atoms at given positions, the packed tables of
``KSHamiltonian.set_projectors``: projector.hpp:38-101 puts the functions beta_i(|r - R|) Y_lm(r - R)
on the atom's sphere (spherical_grid.hpp:59-160) in the order (beta i, m), and couples two functions
by D_ij when their m index agrees (kb_coeff, projector.hpp:88-96).  The device kernels take at most
four functions per projector, so an atom's functions are packed into groups of at most four, each a
projector of its own on the same sphere; functions coupled by D_ij (same l and m, any radial index)
always share a group, so every group's 4 x 4 KB block is exact and the groups add up to the
reference's operator.  An atom with n functions costs ceil(n / 4) gathers of its sphere.
"""

from __future__ import annotations

import gzip
import re
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Pseudopotential:
    element: str
    z_valence: float
    r: np.ndarray                  # radial mesh (bohr)
    rab: np.ndarray                # dr / di of the mesh
    vlocal: np.ndarray             # local potential on the mesh (Hartree)
    beta_l: list = field(default_factory=list)        # angular momentum of each radial projector
    beta: list = field(default_factory=list)          # beta_i(r) on the mesh
    beta_cutoff: list = field(default_factory=list)   # mesh index where each beta ends
    dij: np.ndarray = field(default_factory=lambda: np.zeros((0, 0)))   # KB coefficients (Hartree)

    def num_projectors_l(self) -> int:
        return len(self.beta_l)

    def num_projectors_lm(self) -> int:
        return int(sum(2 * l + 1 for l in self.beta_l))

    def projector_radius(self) -> float:
        """Radius beyond which every projector vanishes (the largest cutoff of the PP_BETA blocks)."""
        if not self.beta_cutoff:
            return 0.0
        return float(max(self.r[min(c, len(self.r) - 1)] for c in self.beta_cutoff))

    def lm_functions(self):
        """(beta index, l, m index 0..2l) of every projector function, in the reference's order."""
        out = []
        for i, l in enumerate(self.beta_l):
            for mm in range(2 * l + 1):
                out.append((i, l, mm))
        return out

    def kb_coefficients(self) -> np.ndarray:
        """kb_coeff[ilm][jlm] = D_ij when the two functions have the same m index, else 0
        (projector.hpp:88-96)."""
        fn = self.lm_functions()
        n = len(fn)
        kb = np.zeros((n, n))
        for a, (i, _, mi) in enumerate(fn):
            for b, (j, _, mj) in enumerate(fn):
                if mi == mj:
                    kb[a, b] = self.dij[i, j]
        return kb


# ---------------------------------------------------------------- UPF reading

def _numbers(text: str) -> np.ndarray:
    return np.array([float(x.replace("D", "E").replace("d", "e")) for x in text.split()], dtype=np.float64)


def _read_text(path: str) -> str:
    if path.endswith(".gz"):
        with gzip.open(path, "rt", errors="replace") as f:
            return f.read()
    with open(path, "r", errors="replace") as f:
        return f.read()


def _finish(element, z, r, rab, vloc_ry, betas, dij_ry) -> Pseudopotential:
    beta_l, beta, cut = [], [], []
    for l, rbeta, ci in betas:
        rb = np.zeros_like(r)
        rb[: len(rbeta)] = rbeta[: len(r)]
        b = np.zeros_like(r)
        nz = r > 0
        b[nz] = rb[nz] / r[nz]
        if not nz.all():                 # r = 0 on the mesh: the limit (zero for l > 0)
            i0 = np.where(~nz)[0]
            if l == 0 and len(r) > 2:
                b[i0] = b[i0 + 1] if i0[0] + 1 < len(r) else 0.0
            else:
                b[i0] = 0.0
        # the projector's extent: the file's cutoff index, shortened to the last point where |r beta|
        # is above 1e-10 of its maximum (some files carry a negligible tail to the end of the mesh)
        big = np.nonzero(np.abs(rb) > 1e-10 * max(float(np.max(np.abs(rb))), 1e-300))[0]
        last = int(big[-1]) + 1 if len(big) else 0
        ci = last if (ci is None or ci <= 0) else min(int(ci), last)
        beta_l.append(int(l))
        beta.append(b)
        cut.append(int(ci))
    nb = len(betas)
    d = np.asarray(dij_ry, dtype=np.float64).reshape(nb, nb) * 0.5 if nb else np.zeros((0, 0))
    return Pseudopotential(element.strip(), float(z), r, rab, 0.5 * np.asarray(vloc_ry, dtype=np.float64)[: len(r)],
                           beta_l, beta, cut, d)


def _parse_v2(text: str) -> Pseudopotential:
    # the PP_INFO block may hold unescaped text; drop it before parsing the XML
    text = re.sub(r"<PP_INFO>.*?</PP_INFO>", "", text, flags=re.S)
    text = text.replace("&", "&amp;")
    root = ET.fromstring(text[text.index("<UPF"):])
    head = root.find("PP_HEADER").attrib
    element = head.get("element", "")
    z = float(head.get("z_valence", "0"))
    mesh = root.find("PP_MESH")
    r = _numbers(mesh.find("PP_R").text)
    rab = _numbers(mesh.find("PP_RAB").text)
    vloc = _numbers(root.find("PP_LOCAL").text) if root.find("PP_LOCAL") is not None else np.zeros_like(r)
    nl = root.find("PP_NONLOCAL")
    betas, dij = [], []
    if nl is not None:
        blocks = sorted((c for c in nl if c.tag.startswith("PP_BETA")), key=lambda c: int(c.tag.split(".")[1]))
        for c in blocks:
            ci = c.attrib.get("cutoff_radius_index")
            betas.append((int(c.attrib["angular_momentum"]), _numbers(c.text), int(ci) if ci else None))
        d = nl.find("PP_DIJ")
        if d is not None and betas:
            dij = _numbers(d.text)
    return _finish(element, z, r, rab, vloc, betas, dij if len(betas) else [])


def _block(text: str, tag: str) -> str:
    m = re.search(r"<%s[^>]*>(.*?)</%s>" % (re.escape(tag), re.escape(tag)), text, flags=re.S)
    return m.group(1) if m else ""


def _parse_v1(text: str) -> Pseudopotential:
    head = _block(text, "PP_HEADER").strip().splitlines()
    element = head[1].split()[0] if len(head) > 1 else ""
    z = 0.0
    nbeta = 0
    for line in head:
        low = line.lower()
        if "z valence" in low:
            z = float(line.split()[0].replace("D", "E"))
        if "number of wavefunctions, number of projectors" in low or "wavefunctions, projectors" in low:
            nbeta = int(line.split()[1])
    r = _numbers(_block(text, "PP_R"))
    rab = _numbers(_block(text, "PP_RAB"))
    vloc = _numbers(_block(text, "PP_LOCAL"))
    nl = _block(text, "PP_NONLOCAL")
    betas = []
    for m in re.finditer(r"<PP_BETA>(.*?)</PP_BETA>", nl, flags=re.S):
        lines = m.group(1).strip().splitlines()
        l = int(lines[0].split()[1])
        npts = int(lines[1].split()[0])
        vals = _numbers(" ".join(lines[2:]))[:npts]
        betas.append((l, vals, npts - 1))
    nbeta = len(betas) or nbeta
    dij = np.zeros((nbeta, nbeta))
    dl = _block(nl, "PP_DIJ").strip().splitlines()
    if dl:
        nnz = int(dl[0].split()[0])
        for line in dl[1:1 + nnz]:
            i, j, v = line.split()[:3]
            dij[int(i) - 1, int(j) - 1] = float(v.replace("D", "E"))
            dij[int(j) - 1, int(i) - 1] = float(v.replace("D", "E"))
    return _finish(element, z, r, rab, vloc, betas, dij)


def read_upf(path: str) -> Pseudopotential:
    """A UPF file (version 1 or 2, optionally gzip-compressed)."""
    text = _read_text(path)
    if "<UPF" in text[:2000] or 'version="2' in text[:2000]:
        return _parse_v2(text)
    return _parse_v1(text)


def write_upf(path: str, ps: Pseudopotential):
    """A UPF version 2 file holding ``ps`` (energies back in Rydberg, PP_BETA as r * beta(r))."""
    def arr(tag, v, extra=""):
        body = "\n".join(" ".join(f"{x:.16e}" for x in v[i:i + 4]) for i in range(0, len(v), 4))
        return f'<{tag} type="real" size="{len(v)}" columns="4"{extra}>\n{body}\n</{tag}>\n'
    nb = len(ps.beta_l)
    out = ['<UPF version="2.0.1">\n',
           f'<PP_HEADER element="{ps.element}" pseudo_type="NC" z_valence="{ps.z_valence:.16e}" '
           f'l_max="{max(ps.beta_l, default=-1)}" mesh_size="{len(ps.r)}" number_of_proj="{nb}"/>\n',
           "<PP_MESH>\n", arr("PP_R", ps.r), arr("PP_RAB", ps.rab), "</PP_MESH>\n",
           arr("PP_LOCAL", 2.0 * ps.vlocal), "<PP_NONLOCAL>\n"]
    for i, l in enumerate(ps.beta_l):
        out.append(arr(f"PP_BETA.{i + 1}", ps.r * ps.beta[i],
                       f' index="{i + 1}" angular_momentum="{l}" cutoff_radius_index="{ps.beta_cutoff[i]}"'))
    if nb:
        out.append(arr("PP_DIJ", (2.0 * ps.dij).reshape(-1)))
    out.append("</PP_NONLOCAL>\n</UPF>\n")
    with open(path, "w") as f:
        f.write("".join(out))


# ---------------------------------------------------------------- projectors from pseudopotentials

_Y00 = 0.5 / np.sqrt(np.pi)


def real_ylm(l: int, xyz: np.ndarray) -> np.ndarray:
    """Real spherical harmonics Y_lm, m = -l..l, at cartesian offsets xyz [n, 3] (zero at the origin
    for l > 0); rows [2l + 1, n].  l = 1 is (y, z, x) sqrt(3 / 4 pi) / r, the convention of the
    synthetic projectors; l = 2, 3 the usual real (tesseral) harmonics without the Condon-Shortley phase."""
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    r2 = x * x + y * y + z * z
    r = np.sqrt(r2)
    on = r > 0
    inv = np.where(on, 1.0 / np.where(on, r, 1.0), 0.0)
    if l == 0:
        return np.full((1, len(x)), _Y00)
    if l == 1:
        c = np.sqrt(3.0 / (4.0 * np.pi))
        return np.stack([c * y * inv, c * z * inv, c * x * inv])
    if l == 2:
        i2 = inv * inv
        c1 = 0.5 * np.sqrt(15.0 / np.pi)
        return np.stack([c1 * x * y * i2, c1 * y * z * i2, 0.25 * np.sqrt(5.0 / np.pi) * (3 * z * z - r2) * i2,
                         c1 * x * z * i2, 0.25 * np.sqrt(15.0 / np.pi) * (x * x - y * y) * i2])
    if l == 3:
        i3 = inv * inv * inv
        a = 0.25 * np.sqrt(35.0 / (2 * np.pi))
        b = 0.5 * np.sqrt(105.0 / np.pi)
        c = 0.25 * np.sqrt(21.0 / (2 * np.pi))
        d = 0.25 * np.sqrt(7.0 / np.pi)
        return np.stack([a * y * (3 * x * x - y * y) * i3, b * x * y * z * i3, c * y * (5 * z * z - r2) * i3,
                         d * z * (5 * z * z - 3 * r2) * i3, c * x * (5 * z * z - r2) * i3,
                         0.5 * b * z * (x * x - y * y) * i3, a * x * (x * x - 3 * y * y) * i3])
    raise ValueError("projectors up to l = 3 are supported")


RADIAL_DR = 0.002   # spacing (bohr) of the uniform radial tables


def radial_tables(ps: Pseudopotential, dr: float = RADIAL_DR) -> np.ndarray:
    """Every beta_i resampled on the uniform grid r_k = k dr up to the projector radius (a cubic spline
    through the file's mesh points up to each projector's end, zero beyond): [nbeta, nr].  The host
    and the device evaluate projectors from these tables with the same cubic convolution."""
    from scipy.interpolate import CubicSpline
    cache = getattr(ps, "_tables", None)
    if cache is not None and cache[0] == dr:
        return cache[1]
    nr = int(np.ceil(ps.projector_radius() / dr)) + 3
    rk = np.arange(nr) * dr
    out = np.zeros((len(ps.beta_l), nr))
    for i in range(len(ps.beta_l)):
        c = min(ps.beta_cutoff[i] + 2, len(ps.r))
        rr, bb = ps.r[:c], ps.beta[i][:c]
        keep = np.concatenate([[True], np.diff(rr) > 0])
        sp = CubicSpline(rr[keep], bb[keep], extrapolate=False)
        out[i] = np.nan_to_num(sp(rk), nan=0.0)
        out[i][rk > rr[-1]] = 0.0
    ps._tables = (dr, out)
    return out


def radial_eval(table: np.ndarray, dr: float, l: int, d: np.ndarray) -> np.ndarray:
    """Cubic convolution (Catmull-Rom) on the uniform table at distances d; the point before r = 0
    mirrors the table with the parity of r^l, points past the end are zero."""
    d = np.asarray(d, dtype=np.float64)
    nr = len(table)
    x = d / dr
    k = np.floor(x).astype(np.int64)
    t = x - k
    sgn = -1.0 if l % 2 else 1.0

    def f(i):
        v = np.where((i >= 0) & (i < nr), table[np.clip(i, 0, nr - 1)], 0.0)
        return np.where(i < 0, sgn * table[np.clip(-i, 0, nr - 1)], v)

    fm, f0, f1, f2 = f(k - 1), f(k), f(k + 1), f(k + 2)
    val = 0.5 * (2.0 * f0 + (f1 - fm) * t + (2.0 * fm - 5.0 * f0 + 4.0 * f1 - f2) * t * t
                 + (3.0 * f0 - fm - 3.0 * f1 + f2) * t * t * t)
    return np.where(k < nr, val, 0.0)


def _radial(ps: Pseudopotential, i: int, d: np.ndarray) -> np.ndarray:
    """beta_i at distances d (the uniform table and its cubic convolution)."""
    return radial_eval(radial_tables(ps)[i], RADIAL_DR, ps.beta_l[i], d)


def group_functions(ps: Pseudopotential, width: int = 4):
    """Packs the (beta, m) functions into groups of at most ``width``; the functions D_ij couples (same
    l and m index, any radial index) stay together.  Returns lists of function indices."""
    fn = ps.lm_functions()
    classes = {}
    for k, (i, l, mm) in enumerate(fn):
        classes.setdefault((l, mm), []).append(k)
    cls = sorted(classes.values(), key=len, reverse=True)
    if any(len(c) > width for c in cls):
        raise ValueError(f"more than {width} coupled projector functions in one (l, m) channel")
    groups = []
    for c in cls:                      # first fit, largest classes first
        for g in groups:
            if len(g) + len(c) <= width:
                g.extend(c)
                break
        else:
            groups.append(list(c))
    return [sorted(g) for g in groups]


def projector_tables(cell, sizes, atoms):
    """Packed tables for ``KSHamiltonian.set_projectors`` from ``atoms`` = [(Pseudopotential, cartesian
    position)]: one projector per group of at most four functions of an atom, all on the atom's sphere of
    radius ``projector_radius``.  Returns (points, positions, matrices, coeff, npts, nlm, owner), owner[p]
    being the atom index of projector p."""
    from .core import spherical_grid
    lat = np.asarray(cell.lattice, dtype=np.float64)
    rows = []
    for ia, (ps, pos) in enumerate(atoms):
        if ps.num_projectors_lm() == 0:
            continue
        pts, dist, rel = spherical_grid(cell, sizes, np.asarray(pos, dtype=np.float64), ps.projector_radius())
        xyz = rel.astype(np.float64) @ lat           # contravariant offsets to cartesian
        d = dist.astype(np.float64)
        fn = ps.lm_functions()
        vals = np.zeros((len(fn), len(d)))
        k = 0
        for i, l in enumerate(ps.beta_l):
            rad = _radial(ps, i, d)
            y = real_ylm(l, xyz)
            for mm in range(2 * l + 1):
                vals[k] = rad * y[mm]
                k += 1
        kb = ps.kb_coefficients()
        for g in group_functions(ps):
            rows.append((ia, pts, rel, vals[g], kb[np.ix_(g, g)]))
    nproj = len(rows)
    maxsph = max((len(r[1]) for r in rows), default=0)
    points = np.full((nproj, maxsph, 3), -1, np.int32)
    positions = np.zeros((nproj, maxsph, 3), np.float32)
    matrices = np.zeros((nproj, 4, maxsph))
    coeff = np.zeros((nproj, 4, 4))
    npts = np.zeros(nproj, np.int32)
    nlm = np.zeros(nproj, np.int32)
    owner = np.zeros(nproj, np.int32)
    for p, (ia, pts, rel, v, kbg) in enumerate(rows):
        n = len(pts)
        points[p, :n] = pts
        positions[p, :n] = rel
        matrices[p, : len(v), :n] = v
        coeff[p, : len(v), : len(v)] = kbg
        npts[p] = n
        nlm[p] = len(v)
        owner[p] = ia
    return points, positions, matrices, coeff, npts, nlm, owner


# ---------------------------------------------------------------- local potential

def _erf(x):
    from scipy.special import erf
    return erf(x)


def local_potential(cell, sizes, atoms, sigma: float | None = None, tolerance: float = 1e-10) -> np.ndarray:
    """The ions' local potential on the grid (Hartree), [nx, ny, nz].

    Each atom's V_loc(r), whose tail is -Z/r, is split as in hamiltonian/atomic_potential.hpp:117-200
    into a short-range part V_sr(r) = V_loc(r) + Z erf(r / sigma) / r, summed on the atom's sphere
    (spline through the mesh, out to where |V_sr| falls below ``tolerance``), and the potential of a
    Gaussian charge Z of width sigma, -Z erf(r / sigma) / r, summed over all periodic images in Fourier
    space: V(G) = -4 pi Z exp(-G^2 sigma^2 / 4) / (Omega G^2) e^{-i G.R}, G = 0 dropped (the neutralising
    background of a periodic cell, as the Poisson solver of the Hartree term drops it); the constant
    that leaves is set so the grid average is sum_atoms alpha_Z / Omega, alpha_Z = int (V_loc + Z/r)
    d^3 r, whatever sigma is.  The default
    sigma, 3.1 grid spacings, keeps exp(-G^2 sigma^2 / 4) below 1e-10 at the grid's largest G, so the
    Fourier sum of the Gaussian part is not truncated."""
    from scipy.interpolate import CubicSpline
    from .core import spherical_grid
    lat = np.asarray(cell.lattice, dtype=np.float64)
    n = tuple(int(v) for v in sizes)
    if sigma is None:
        sigma = 3.1 * max(np.linalg.norm(lat[i]) / n[i] for i in range(3))
    npoint = int(np.prod(n))
    V = np.zeros(npoint)
    rec = 2.0 * np.pi * np.linalg.inv(lat).T              # rows b_i, a_i . b_j = 2 pi delta_ij
    omega = abs(np.linalg.det(lat))
    # long range: Gaussian charges in Fourier space
    m = [np.fft.fftfreq(k, 1.0 / k) for k in n]
    M = np.stack(np.meshgrid(*m, indexing="ij"), axis=-1)   # integer frequencies
    G = M @ rec
    g2 = np.sum(G * G, axis=-1)
    rho = np.zeros(n, dtype=np.complex128)
    for ps, R in atoms:
        rho += ps.z_valence * np.exp(-1j * (G @ np.asarray(R, dtype=np.float64)))
    with np.errstate(divide="ignore", invalid="ignore"):
        vg = np.where(g2 > 0, -4.0 * np.pi * rho * np.exp(-g2 * sigma * sigma / 4.0) / (omega * np.where(g2 > 0, g2, 1.0)), 0.0)
    V += np.real(np.fft.ifftn(vg) * npoint).reshape(-1)
    # the sphere sums below carry the mean of V_sr, (alpha_Z - pi Z sigma^2) / Omega per atom with
    # alpha_Z = int (V_loc + Z / r) d^3 r; adding pi Z sigma^2 / Omega leaves the G = 0 term at the
    # pseudopotential's own alpha_Z, independent of the split
    V += sum(np.pi * ps.z_valence * sigma * sigma for ps, _ in atoms) / omega
    # short range: spheres
    for ps, R in atoms:
        r = ps.r
        with np.errstate(divide="ignore", invalid="ignore"):
            tail = np.where(r > 0, ps.z_valence * _erf(r / sigma) / np.where(r > 0, r, 1.0),
                            ps.z_valence * 2.0 / (np.sqrt(np.pi) * sigma))
        vsr = ps.vlocal + tail
        big = np.nonzero(np.abs(vsr) > tolerance)[0]
        if not len(big):
            continue
        last = min(int(big[-1]) + 2, len(r) - 1)
        keep = np.concatenate([[True], np.diff(r[: last + 1]) > 0])
        sp = CubicSpline(r[: last + 1][keep], vsr[: last + 1][keep], extrapolate=False)
        pts, dist, _ = spherical_grid(cell, sizes, np.asarray(R, dtype=np.float64), float(r[last]))
        vals = np.nan_to_num(sp(dist.astype(np.float64)), nan=0.0)
        flat = (pts[:, 0].astype(np.int64) * n[1] + pts[:, 1]) * n[2] + pts[:, 2]
        np.add.at(V, flat, vals)
    return V.reshape(n)


def set_ions(ham, atoms, sigma: float | None = None, device: bool = False):
    """The local potential and the nonlocal projectors of ``atoms`` = [(Pseudopotential, cartesian
    position)] on a KSHamiltonian (its basis's cell and grid); returns the local potential.  With
    ``device`` the projector tables are built by the device kernels from the same uniform radial
    tables and groups (the same projectors, in the same order, as ``projector_tables``), and
    ``ham.move_atoms`` later rebuilds them on the device for new positions."""
    basis = ham.basis
    cell, sizes = basis.cell, tuple(basis.sizes)
    V = local_potential(cell, sizes, atoms, sigma)
    ham.set_scalar_potential(V)
    if device:
        build_radial_device(ham, atoms)
    else:
        points, pos, mats, coeff, npts, nlm, _ = projector_tables(cell, sizes, atoms)
        ham.set_projectors(points, pos, mats, coeff, npts, nlm)
    return V


def build_radial_device(ham, atoms):
    """The projectors of ``atoms`` built on the device (``inqb_projectors_build_radial``)."""
    import ctypes as C
    from . import _lib
    species, index = [], {}
    for ps, _ in atoms:
        if id(ps) not in index:
            index[id(ps)] = len(species)
            species.append(ps)
    tabs = [radial_tables(ps) for ps in species]
    nr = max([t.shape[1] for t in tabs] + [1])
    rows, fn, kb, ngroups, radius = [], [], [], [], []
    for ps, t in zip(species, tabs):
        base = len(rows)
        for row in t:
            rows.append(np.pad(row, (0, nr - len(row))))
        groups = group_functions(ps) if ps.num_projectors_lm() else []
        kbf = ps.kb_coefficients()
        lmf = ps.lm_functions()
        for g in groups:
            f = np.full((4, 3), -1, np.int32)
            f[:, 1:] = 0
            blk = np.zeros((4, 4))
            for j, k in enumerate(g):
                i, l, mm = lmf[k]
                f[j] = (base + i, l, mm)
            blk[: len(g), : len(g)] = kbf[np.ix_(g, g)]
            fn.append(f)
            kb.append(blk)
        ngroups.append(len(groups))
        radius.append(ps.projector_radius())
    pos = np.ascontiguousarray(np.array([R for _, R in atoms], dtype=np.float64).reshape(-1, 3))
    spc = np.ascontiguousarray([index[id(ps)] for ps, _ in atoms], dtype=np.int32)
    tables = np.ascontiguousarray(np.array(rows, dtype=np.float64).reshape(-1))
    fn_a = np.ascontiguousarray(np.array(fn, dtype=np.int32).reshape(-1))
    kb_a = np.ascontiguousarray(np.array(kb, dtype=np.float64).reshape(-1))
    ng = np.ascontiguousarray(ngroups, dtype=np.int32)
    rad = np.ascontiguousarray(radius, dtype=np.float64)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    dp = lambda a: a.ctypes.data_as(_lib.DP)
    ham.ctx.check(ham.ctx.lib.inqb_projectors_build_radial(
        ham.handle, len(atoms), dp(pos), vp(spc), len(species), dp(rad), int(nr), float(RADIAL_DR), len(rows),
        dp(tables) if len(rows) else None, vp(ng), vp(fn_a) if len(fn) else None, dp(kb_a) if len(kb) else None))
    ham._moving_atoms = len(atoms)
