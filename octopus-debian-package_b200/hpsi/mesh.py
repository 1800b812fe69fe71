"""Real-space mesh construction (host-side set-up, as the Fortran host does it).

The library never builds meshes: it receives the integer coordinates of the
``np`` inner points followed by the ``np_part - np`` boundary points, exactly the
arrays the reference keeps in ``mesh%idx`` after ``mesh_init_stage_2``.  This
module restates that construction so that Python callers (tests, benchmarks)
can produce the same point lists:

* bounding range ``nr``: the largest ``j`` with ``j*h <= bound + 1e-12``
  (src/grid/mesh_init.F90:100-119), symmetric, then enlarged by the stencil
  half-width (src/grid/mesh_init.F90:216-218);
* inner points: every grid point of the (un-enlarged) range inside the box
  (src/grid/mesh_init.F90:261-272), with ``box_sphere`` / ``box_parallelepiped``
  ``contains_point`` semantics (src/boxes/box_sphere.F90:91-104, delta 1e-12,
  src/boxes/box.F90:38);
* boundary points: stencil neighbours of inner points that are neither inner
  nor inside the box, de-duplicated (src/grid/mesh_init.F90:293-329);
* both lists are reordered by the blocked index (``reorder_points``,
  src/grid/mesh_init.F90:786-1055; ``get_blocked_index``,
  src/grid/index.F90:358-394).  The default block size follows the CPU default
  ``StatesBlockSize`` = 4: (80, 4, 10).

Periodic meshes put the images of the boundary points in ``per_inner`` (the
``per_points(POINT_INNER, :)`` array of src/grid/boundaries.F90) so that the
periodic boundary copy (src/grid/boundaries_inc.F90:650-700) can be applied.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .stencil import star_points

BOX_BOUNDARY_DELTA = 1e-12


@dataclass
class Mesh:
    """Point list of one real-space mesh (0-based indices)."""

    lxyz: np.ndarray          # (np_part, 3) int32 grid coordinates
    np: int                   # inner points
    spacing: np.ndarray       # (3,) float64
    periodic: bool = False
    per_inner: np.ndarray | None = None   # (np_part-np,) inner image of each boundary point
    label: str = ""
    extra: dict = field(default_factory=dict)

    @property
    def np_part(self) -> int:
        return int(self.lxyz.shape[0])

    @property
    def x(self) -> np.ndarray:
        """Cartesian coordinates of every point, (np_part, 3)."""
        return self.lxyz.astype(np.float64) * self.spacing[None, :]

    @property
    def vol_pp(self) -> float:
        return float(np.prod(self.spacing))


def blocked_index(points: np.ndarray, offset: np.ndarray, bsize, nblocks) -> np.ndarray:
    """``get_blocked_index`` with x fastest, for an (n, 3) array of points."""
    p = points.astype(np.int64) + offset[None, :].astype(np.int64)
    bsize = np.asarray(bsize, dtype=np.int64)
    nblocks = np.asarray(nblocks, dtype=np.int64)
    j_local = np.zeros(len(p), dtype=np.int64)
    j_block = np.zeros(len(p), dtype=np.int64)
    sl = 1
    sb = 1
    for d in range(3):
        j_local += (p[:, d] % bsize[d]) * sl
        sl *= bsize[d]
        j_block += (p[:, d] // bsize[d]) * sb
        sb *= nblocks[d]
    return j_local + j_block * int(np.prod(bsize))


def _build(inner_lo, inner_hi, contains, spacing, order, bsize, periodic=False):
    """Generic builder over the inner index range [inner_lo, inner_hi] (inclusive)."""
    spacing = np.broadcast_to(np.asarray(spacing, dtype=np.float64), (3,)).copy()
    inner_lo = np.asarray(inner_lo, dtype=np.int64)
    inner_hi = np.asarray(inner_hi, dtype=np.int64)
    ax = [np.arange(inner_lo[d], inner_hi[d] + 1) for d in range(3)]
    gz, gy, gx = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    cand = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)
    inside = contains(cand.astype(np.float64) * spacing[None, :])
    inner = cand[inside]

    enlarge = order
    nr_lo = inner_lo - enlarge
    nr_hi = inner_hi + enlarge
    ext = nr_hi - nr_lo + 1
    # dense lookup over the enlarged range: -1 = not inner
    lut = -np.ones(ext[::-1], dtype=np.int64)
    ii = inner - nr_lo[None, :]
    lut[ii[:, 2], ii[:, 1], ii[:, 0]] = np.arange(len(inner))

    pts = star_points(order)
    nb = (inner[:, None, :] + pts[None, :, :]).reshape(-1, 3)
    jj = nb - nr_lo[None, :]
    is_inner = lut[jj[:, 2], jj[:, 1], jj[:, 0]] >= 0
    cand_b = nb[~is_inner]
    if len(cand_b):
        in_box = contains(cand_b.astype(np.float64) * spacing[None, :])
        cand_b = cand_b[~in_box]
    bnd = np.unique(cand_b, axis=0) if len(cand_b) else np.zeros((0, 3), dtype=np.int64)

    offset = ext // 2
    nblocks = ext // np.asarray(bsize) + 1
    inner = inner[np.argsort(blocked_index(inner, offset, bsize, nblocks), kind="stable")]
    if len(bnd):
        bnd = bnd[np.argsort(blocked_index(bnd, offset, bsize, nblocks), kind="stable")]
    lxyz = np.ascontiguousarray(np.concatenate([inner, bnd]).astype(np.int32))
    mesh = Mesh(lxyz=lxyz, np=len(inner), spacing=spacing, periodic=periodic)
    if periodic:
        n = inner_hi - inner_lo + 1
        img = (bnd - inner_lo[None, :]) % n[None, :] + inner_lo[None, :]
        lut2 = -np.ones(ext[::-1], dtype=np.int64)
        ii = inner - nr_lo[None, :]
        lut2[ii[:, 2], ii[:, 1], ii[:, 0]] = np.arange(len(inner))
        jj = img - nr_lo[None, :]
        mesh.per_inner = np.ascontiguousarray(lut2[jj[:, 2], jj[:, 1], jj[:, 0]].astype(np.int32))
        assert (mesh.per_inner >= 0).all()
    return mesh


def _nr(bound: float, h: float) -> int:
    jj = 0
    while True:
        jj += 1
        if jj * h > bound + BOX_BOUNDARY_DELTA:
            return jj - 1


def sphere_mesh(radius: float, spacing: float, order: int = 4, bsize=(80, 4, 10),
                center=(0.0, 0.0, 0.0)) -> Mesh:
    """Sphere box of the given radius around ``center`` (``BoxShape = sphere``)."""
    c = np.asarray(center, dtype=np.float64)
    n = _nr(float(np.max(np.abs(c)) + radius), spacing)

    def contains(xyz):
        return np.sum((xyz - c[None, :]) ** 2, axis=1) <= (radius + BOX_BOUNDARY_DELTA) ** 2

    m = _build([-n] * 3, [n] * 3, contains, spacing, order, bsize)
    m.label = f"sphere R={radius} h={spacing}"
    return m


def parallelepiped_mesh(half_length, spacing, order: int = 4, bsize=(80, 4, 10)) -> Mesh:
    """Symmetric finite parallelepiped (``BoxShape = parallelepiped``, ``Lsize``)."""
    L = np.broadcast_to(np.asarray(half_length, dtype=np.float64), (3,))
    n = [_nr(float(L[d]), spacing) for d in range(3)]

    def contains(xyz):
        return np.all(np.abs(xyz) <= L[None, :] + BOX_BOUNDARY_DELTA, axis=1)

    m = _build([-v for v in n], n, contains, spacing, order, bsize)
    m.label = f"parallelepiped L={tuple(L)} h={spacing}"
    return m


def index_box_mesh(shape, spacing, order: int = 4, bsize=(80, 4, 10),
                   periodic: bool = False, origin=None) -> Mesh:
    """A box of exactly ``shape`` = (nx, ny, nz) inner points.

    Points run from ``origin`` (default ``-shape//2``) along each axis, so a 64^3
    box has np = 262,144 and, with the zero boundary, np_part = np + 6*64^2*4.
    With ``periodic`` the boundary points are the periodic images.
    """
    shape = np.asarray(shape, dtype=np.int64)
    lo = -(shape // 2) if origin is None else np.asarray(origin, dtype=np.int64)
    hi = lo + shape - 1
    h = np.broadcast_to(np.asarray(spacing, dtype=np.float64), (3,))

    def contains(xyz):
        ijk = np.rint(xyz / h[None, :]).astype(np.int64)
        return np.all((ijk >= lo[None, :]) & (ijk <= hi[None, :]), axis=1)

    m = _build(lo, hi, contains, spacing, order, bsize, periodic=periodic)
    m.label = f"box {tuple(int(s) for s in shape)} h={spacing}{' periodic' if periodic else ''}"
    return m


def permuted(mesh: Mesh, seed: int = 0) -> tuple[Mesh, np.ndarray, np.ndarray]:
    """Same mesh with inner and boundary points shuffled independently.

    Returns (mesh', perm, inv) where ``mesh'.lxyz = mesh.lxyz[perm]``.  Used to
    show that results do not depend on the point order.
    """
    rng = np.random.default_rng(seed)
    pi = rng.permutation(mesh.np)
    pb = mesh.np + rng.permutation(mesh.np_part - mesh.np)
    perm = np.concatenate([pi, pb])
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    m2 = Mesh(lxyz=np.ascontiguousarray(mesh.lxyz[perm]), np=mesh.np, spacing=mesh.spacing,
              periodic=mesh.periodic, label=mesh.label + " (permuted)")
    if mesh.per_inner is not None:
        # boundary b' = perm[np + b'] - np in the old numbering; its image is old inner index
        old_b = perm[mesh.np:] - mesh.np
        m2.per_inner = np.ascontiguousarray(inv[mesh.per_inner[old_b]].astype(np.int32))
    return m2, perm, inv
