"""Seeded synthetic systems for the benchmark configurations.

There is no public data set for this path; every input is generated here from
a seed (``numpy.random.default_rng``), with the shapes, sizes and value
distributions of the benchmark configurations:

* states: complex Gaussian noise, a 3-point box filter along each axis, then
  Cholesky orthonormalisation (FP64);
* local potential: soft-Coulomb wells -Z / sqrt(|r - R|^2 + 1), Z ~ U[1, 4],
  centres uniform in the inner 60 % of the box;
* KB projectors: per atom 9 projectors (l = 0, 1, 2) p(r) = exp(-r^2/0.8) *
  Y_lm(r) on a 2.0-bohr sphere, KB energies ~ U[-2, 2] Ha, scal = e * vol_pp
  (hamiltonian_elec_base_build_proj, src/hamiltonian/hamiltonian_elec_base.F90:603-634).
  The real spherical harmonics follow the sign convention of src/math/ylm.c
  (l <= 2, Y = 0 at r = 0 for l > 0), with normalisation constants computed
  from their closed forms.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mesh import Mesh, index_box_mesh, sphere_mesh


def dense_lookup(mesh: Mesh, which: str = "inner"):
    """(lut, lo) with lut[z, y, x] = point index or -1 over the bounding box."""
    n = mesh.np if which == "inner" else mesh.np_part
    lx = mesh.lxyz[:n].astype(np.int64)
    lo = lx.min(axis=0)
    ext = lx.max(axis=0) - lo + 1
    lut = -np.ones(ext[::-1], dtype=np.int64)
    ii = lx - lo
    lut[ii[:, 2], ii[:, 1], ii[:, 0]] = np.arange(n)
    return lut, lo


def box_filter(mesh: Mesh, f: np.ndarray, chunk: int = 16) -> np.ndarray:
    """3-point box filter along x, y and z over the inner points (zero outside),
    applied to ``chunk`` states at a time."""
    lut, lo = dense_lookup(mesh)
    ii = mesh.lxyz[: mesh.np].astype(np.int64) - lo
    mask = np.zeros(tuple(s + 2 for s in lut.shape), dtype=bool)
    mask[1:-1, 1:-1, 1:-1][ii[:, 2], ii[:, 1], ii[:, 0]] = True
    f = np.asarray(f)
    cols = f.shape[1:] if f.ndim > 1 else ()
    f2 = f.reshape(f.shape[0], -1)
    out = np.empty((mesh.np, f2.shape[1]), dtype=f2.dtype)
    for c0 in range(0, f2.shape[1], chunk):
        c1 = min(c0 + chunk, f2.shape[1])
        g = np.zeros(mask.shape + (c1 - c0,), dtype=f2.dtype)
        g[1:-1, 1:-1, 1:-1][ii[:, 2], ii[:, 1], ii[:, 0]] = f2[: mesh.np, c0:c1]
        for ax in range(3):
            def sl(a, b):
                return tuple(slice(a, b) if i == ax else slice(None) for i in range(3))
            h = np.zeros_like(g)
            h[sl(1, -1)] = (g[sl(0, -2)] + g[sl(1, -1)] + g[sl(2, None)]) / 3.0
            # keep the zero frame and the region outside the mesh at zero
            h[~mask] = 0
            g = h
        out[:, c0:c1] = g[1:-1, 1:-1, 1:-1][ii[:, 2], ii[:, 1], ii[:, 0]]
    return out.reshape((mesh.np,) + cols)


def orthonormalize(mesh: Mesh, psi: np.ndarray) -> np.ndarray:
    S = mesh.vol_pp * (psi[: mesh.np].conj().T @ psi[: mesh.np])
    L = np.linalg.cholesky(S)
    return np.linalg.solve(L.conj(), psi.T).T


def random_states(mesh: Mesh, nst: int, rng, orthonormal: bool = True) -> np.ndarray:
    """(np_part, nst) complex128; boundary rows are zero."""
    f = rng.standard_normal((mesh.np, nst)) + 1j * rng.standard_normal((mesh.np, nst))
    f = box_filter(mesh, f)
    if orthonormal:
        f = orthonormalize(mesh, f)
    out = np.zeros((mesh.np_part, nst), dtype=np.complex128)
    out[: mesh.np] = f
    return out


def soft_coulomb(mesh: Mesh, rng, nwells: int = 8) -> np.ndarray:
    x = mesh.x[: mesh.np]
    lo, hi = x.min(axis=0), x.max(axis=0)
    c, half = (lo + hi) / 2, (hi - lo) / 2
    v = np.zeros(mesh.np)
    for _ in range(nwells):
        Z = rng.uniform(1.0, 4.0)
        R = c + rng.uniform(-0.6, 0.6, size=3) * half
        v -= Z / np.sqrt(np.sum((x - R) ** 2, axis=1) + 1.0)
    return v


def real_ylm(l: int, m: int, xyz: np.ndarray) -> np.ndarray:
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    r2 = x * x + y * y + z * z
    if l == 0:
        return np.full(len(x), 0.5 / np.sqrt(np.pi))
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.sqrt(r2)
        if l == 1:
            c = np.sqrt(3.0 / (4 * np.pi))
            val = {-1: -c * y / r, 0: c * z / r, 1: -c * x / r}[m]
        elif l == 2:
            c2 = np.sqrt(15.0 / (4 * np.pi))
            c0 = np.sqrt(5.0 / (16 * np.pi))
            c22 = np.sqrt(15.0 / (16 * np.pi))
            val = {-2: c2 * x * y / r2, -1: -c2 * y * z / r2, 0: c0 * (3 * z * z / r2 - 1),
                   1: -c2 * x * z / r2, 2: c22 * (x * x - y * y) / r2}[m]
        else:
            raise ValueError("l <= 2 only")
    return np.where(r2 < 1e-30, 0.0, val)


@dataclass
class ProjectorSet:
    maps: list
    mats: list      # each (npoints, nprojs)
    scals: list
    positions: np.ndarray


def kb_projectors(mesh: Mesh, natoms: int, rng, radius: float = 2.0, min_dist: float = 2.5,
                  place_radius: float = 10.0, box_center=None) -> ProjectorSet:
    x = mesh.x[: mesh.np]
    center = np.zeros(3) if box_center is None else np.asarray(box_center, dtype=np.float64)
    pos = []
    tries = 0
    while len(pos) < natoms:
        tries += 1
        if tries > 100000:
            raise RuntimeError("could not place atoms")
        p = center + rng.uniform(-place_radius, place_radius, size=3)
        if np.linalg.norm(p - center) > place_radius:
            continue
        if all(np.linalg.norm(p - q) >= min_dist for q in pos):
            pos.append(p)
    pos = np.asarray(pos)
    maps, mats, scals = [], [], []
    lm = [(0, 0)] + [(1, m) for m in (-1, 0, 1)] + [(2, m) for m in (-2, -1, 0, 1, 2)]
    for p in pos:
        d = x - p[None, :]
        r2 = np.sum(d * d, axis=1)
        sel = np.nonzero(r2 <= radius * radius)[0].astype(np.int32)
        dd = d[sel]
        rad = np.exp(-r2[sel] / 0.8)
        P = np.stack([rad * real_ylm(l, m, dd) for (l, m) in lm], axis=1)
        e = rng.uniform(-2.0, 2.0, size=len(lm))
        maps.append(sel)
        mats.append(np.ascontiguousarray(P))
        scals.append(e * mesh.vol_pp)
    return ProjectorSet(maps, mats, scals, pos)


@dataclass
class System:
    mesh: Mesh
    v: np.ndarray
    psi: np.ndarray              # (np_part, nst) complex128
    proj: ProjectorSet | None
    name: str


def config0(seed: int = 0, nst: int = 32, n: int = 64) -> System:
    """Plain H.psi: n^3 box, h = 0.25, zero BC, 32 states, 8 soft-Coulomb wells."""
    rng = np.random.default_rng(seed)
    m = index_box_mesh((n, n, n), 0.25)
    v = soft_coulomb(m, rng)
    psi = random_states(m, nst, rng)
    return System(m, v, psi, None, f"box{n}^3 h=0.25 nst={nst}")


def config1(seed: int = 1, nst: int = 128, radius: float = 12.0, spacing: float = 0.2, natoms: int = 32,
            place_radius: float = 10.0) -> System:
    """Full H.psi with KB: sphere R=12, h=0.2, 32 atoms x 9 projectors, 128 states."""
    rng = np.random.default_rng(seed)
    m = sphere_mesh(radius, spacing)
    v = soft_coulomb(m, rng)
    proj = kb_projectors(m, natoms, rng, place_radius=place_radius)
    psi = random_states(m, nst, rng)
    return System(m, v, psi, proj, f"sphere R={radius} h={spacing} nst={nst} atoms={natoms}")


def config3(seed: int = 2024, nsys: int = 64):
    """Uneven batch of independent systems: cubic boxes with sides
    ~ round-down(exp(U[ln 32, ln 96])), h = 0.25, states per system
    ~ exp(U[ln 4, ln 64]), 2..16 KB atoms each with the config-1 projectors,
    soft-Coulomb wells; states are normalised complex Gaussian noise on the
    inner points.  Returns a list of System (psi holds np_part rows, zero
    boundary rows, ld = nst rounded up to a multiple of 8)."""
    rng = np.random.default_rng(seed)
    sides = np.exp(rng.uniform(np.log(32), np.log(96), nsys)).astype(int)
    nsts = np.exp(rng.uniform(np.log(4), np.log(64), nsys)).astype(int)
    atoms = rng.integers(2, 17, nsys)
    out = []
    for i in range(nsys):
        n = int(sides[i])
        m = index_box_mesh((n, n, n), 0.25)
        v = soft_coulomb(m, rng)
        proj = kb_projectors(m, int(atoms[i]), rng, radius=2.0, min_dist=2.0, place_radius=0.45 * n * 0.25)
        nst = int(nsts[i])
        ld = 8 * ((nst + 7) // 8)
        psi = np.zeros((m.np_part, ld), dtype=np.complex128)
        f = rng.standard_normal((m.np, nst)) + 1j * rng.standard_normal((m.np, nst))
        psi[: m.np, :nst] = f / np.sqrt(m.np * m.vol_pp)
        s = System(m, v, psi, proj, f"box{n}^3 h=0.25 nst={nst} atoms={int(atoms[i])}")
        s.nst = nst
        out.append(s)
    return out
