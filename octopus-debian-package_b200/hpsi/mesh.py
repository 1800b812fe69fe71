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

    # boundary candidates: star neighbours of inner points that are not inner
    # points, marked on the dense enlarged grid (each point once)
    pts = star_points(order)
    inner_mask = lut >= 0
    reach = np.zeros_like(inner_mask)
    for p in pts:
        if not p.any():
            continue
        dx, dy, dz = (int(c) for c in p)
        reach[max(dz, 0): ext[2] + min(dz, 0), max(dy, 0): ext[1] + min(dy, 0), max(dx, 0): ext[0] + min(dx, 0)] |= \
            inner_mask[max(-dz, 0): ext[2] - max(dz, 0), max(-dy, 0): ext[1] - max(dy, 0),
                       max(-dx, 0): ext[0] - max(dx, 0)]
    zz, yy, xx = np.nonzero(reach & ~inner_mask)
    cand_b = np.stack([xx, yy, zz], axis=1).astype(np.int64) + nr_lo[None, :]
    if len(cand_b):
        in_box = contains(cand_b.astype(np.float64) * spacing[None, :])
        cand_b = cand_b[~in_box]
    bnd = cand_b if len(cand_b) else np.zeros((0, 3), dtype=np.int64)

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


# ---------------------------------------------------------------------------
# Mesh order on disk: the restart file indices.obf

from .obf import TYPE_INT_32 as IO_TYPE_INT_32  # noqa: E402,F401
from .obf import TYPE_INT_64 as IO_TYPE_INT_64  # noqa: E402,F401
from .obf import write_obf  # noqa: E402


def cubic_extent(mesh: Mesh) -> np.ndarray:
    """Half-width of the enlarged index range per axis, nr(2, :) (the range
    is symmetric, -nr..nr).  For meshes built here it is the largest |coordinate|
    over inner and boundary points, which is the reference's enlarged range
    (src/grid/mesh_init.F90:216-218) for sphere and parallelepiped boxes."""
    return np.max(np.abs(np.asarray(mesh.lxyz, dtype=np.int64)), axis=0)


def cubic_index(lxyz, extent) -> np.ndarray:
    """Spatial index of IDX_CUBIC (the default MeshIndexType,
    src/grid/mesh_init.F90:232): sum_d (x_d + offset_d) * stride_d with
    offset = grid size // 2 (:234-235) and strides 1, G1, G1*G2 over the
    enlarged grid sizes G = 2 * extent + 1 (:172-175;
    index_point_to_cubic, src/grid/index.F90:313-329)."""
    L = np.asarray(lxyz, dtype=np.int64)
    G = 2 * np.asarray(extent, dtype=np.int64) + 1
    off = G // 2
    if np.any(np.abs(L) > np.asarray(extent)[None, :]):
        raise ValueError("cubic_index: a point lies outside the index range")
    stride = np.array([1, G[0], G[0] * G[1]], dtype=np.int64)
    return ((L + off[None, :]) * stride[None, :]).sum(axis=1)


def cubic_point(index, extent) -> np.ndarray:
    """Inverse of ``cubic_index`` (index_cubic_to_point,
    src/grid/index.F90:295-311): (n, 3) int32 coordinates."""
    t = np.asarray(index, dtype=np.int64).copy()
    G = 2 * np.asarray(extent, dtype=np.int64) + 1
    off = G // 2
    stride = np.array([1, G[0], G[0] * G[1]], dtype=np.int64)
    out = np.empty((t.shape[0], 3), dtype=np.int64)
    for d in (2, 1):
        out[:, d] = t // stride[d] - off[d]
        t = t % stride[d]
    out[:, 0] = t - off[0]
    return out.astype(np.int32)


def hilbert_bits(extent) -> int:
    """Bits per axis of the Hilbert index, idx%bits = max over axes of
    ceil(log2(grid size)) (src/grid/mesh_init.F90:242-243), in integer
    arithmetic (grid sizes 2 * extent + 1 are odd, never a power of two)."""
    G = 2 * np.asarray(extent, dtype=np.int64) + 1
    return int(max(int(g - 1).bit_length() for g in G))


def _hilbert_pack(X, bits):
    # bit b of axis d goes to bit b * 3 + (2 - d) of the index (the bit order of
    # TransposetoInt, src/grid/hilbert.c:94-108)
    h = np.zeros(X.shape[0], dtype=np.int64)
    for b in range(bits):
        for d in range(3):
            h |= ((X[:, d] >> b) & 1) << (b * 3 + 2 - d)
    return h


def _hilbert_unpack(h, bits):
    X = np.zeros((h.shape[0], 3), dtype=np.int64)
    for b in range(bits):
        for d in range(3):
            X[:, d] |= ((h >> (b * 3 + 2 - d)) & 1) << b
    return X


def hilbert_index(lxyz, extent) -> np.ndarray:
    """Spatial index of IDX_HILBERT (MeshIndexType = idx_hilbert,
    index_point_to_hilbert, src/grid/index.F90:343-354): the point shifted by
    the offset, then J. Skilling's axes -> transposed Hilbert index
    ("Programming the Hilbert curve", AIP Conf. Proc. 707, 381 (2004)), the
    algorithm src/grid/hilbert.c uses, vectorised over points."""
    L = np.asarray(lxyz, dtype=np.int64)
    e = np.asarray(extent, dtype=np.int64)
    if np.any(np.abs(L) > e[None, :]):
        raise ValueError("hilbert_index: a point lies outside the index range")
    bits = hilbert_bits(e)
    X = L + ((2 * e + 1) // 2)[None, :]
    # undo the rotations and reflections, from the top bit down
    q = 1 << (bits - 1)
    while q > 1:
        p = q - 1
        for d in range(3):
            hit = (X[:, d] & q) != 0
            X[hit, 0] ^= p
            t = np.where(hit, 0, (X[:, 0] ^ X[:, d]) & p)
            X[:, 0] ^= t
            X[:, d] ^= t
        q >>= 1
    # Gray encode
    for d in (1, 2):
        X[:, d] ^= X[:, d - 1]
    t = np.zeros(X.shape[0], dtype=np.int64)
    q = 1 << (bits - 1)
    while q > 1:
        t ^= np.where((X[:, 2] & q) != 0, q - 1, 0)
        q >>= 1
    X ^= t[:, None]
    return _hilbert_pack(X, bits)


def hilbert_point(index, extent) -> np.ndarray:
    """Inverse of ``hilbert_index`` (index_hilbert_to_point,
    src/grid/index.F90:332-341): (n, 3) int32 coordinates."""
    e = np.asarray(extent, dtype=np.int64)
    bits = hilbert_bits(e)
    X = _hilbert_unpack(np.asarray(index, dtype=np.int64), bits)
    # Gray decode
    t = X[:, 2] >> 1
    for d in (2, 1):
        X[:, d] ^= X[:, d - 1]
    X[:, 0] ^= t
    # redo the rotations and reflections, from the bottom bit up
    q = 2
    while q != (2 << (bits - 1)):
        p = q - 1
        for d in (2, 1, 0):
            hit = (X[:, d] & q) != 0
            X[hit, 0] ^= p
            t = np.where(hit, 0, (X[:, 0] ^ X[:, d]) & p)
            X[:, 0] ^= t
            X[:, d] ^= t
        q <<= 1
    return (X - ((2 * e + 1) // 2)[None, :]).astype(np.int32)


def spatial_index(lxyz, extent, index_type: str = "cubic") -> np.ndarray:
    """Spatial index of the points for MeshIndexType idx_cubic (the default)
    or idx_hilbert."""
    if index_type == "cubic":
        return cubic_index(lxyz, extent)
    if index_type == "hilbert":
        return hilbert_index(lxyz, extent)
    raise ValueError(f"unknown index type {index_type!r}")


def spatial_point(index, extent, index_type: str = "cubic") -> np.ndarray:
    if index_type == "cubic":
        return cubic_point(index, extent)
    if index_type == "hilbert":
        return hilbert_point(index, extent)
    raise ValueError(f"unknown index type {index_type!r}")


def write_indices_obf(path, mesh: Mesh, extent=None, index_type: str = "cubic") -> None:
    """Write the mesh order as the reference's restart file indices.obf
    (index_dump, src/grid/index.F90:176-200): the io_binary header
    (src/basic/io_binary.c:112-150: "pulpo", version 0, the value one in four
    formats for the endianness check, np, type) and the np_part spatial
    indices as int64, in mesh order."""
    idx = spatial_index(mesh.lxyz, cubic_extent(mesh) if extent is None else extent, index_type)
    write_obf(path, idx.astype(np.int64))


def read_indices_obf(path) -> np.ndarray:
    """Spatial indices of an indices.obf file (index_load,
    src/grid/index.F90:204-257, through io_binary_read; header checks and
    byte order in ``hpsi.obf.read_obf``); int32 and int64 payloads are
    accepted."""
    from .obf import read_obf
    v = read_obf(path)
    if v.dtype.kind != "i":
        raise ValueError(f"indices.obf: payload type {v.dtype} is not an integer type")
    return v.astype(np.int64)


def mesh_from_indices_obf(path, np_inner: int, spacing, extent, index_type: str = "cubic") -> Mesh:
    """Mesh point list in the order a reference run stored: the first
    ``np_inner`` entries are the inner points, the rest the boundary points
    (mesh%np_global of the same run)."""
    idx = read_indices_obf(path)
    if not 0 < np_inner <= idx.shape[0]:
        raise ValueError("mesh_from_indices_obf: np_inner outside 1..np_part")
    return Mesh(lxyz=spatial_point(idx, extent, index_type), np=int(np_inner),
                spacing=np.asarray(spacing, dtype=np.float64) * np.ones(3), label=str(path))


def index_checksum(indices) -> int:
    """mesh%idx%checksum: sum over points of (position, 1-based) x spatial
    index in wrapping 64-bit arithmetic (checksum_calculate,
    src/math/checksum.c:30-41, called at src/grid/mesh_init.F90:446)."""
    v = np.asarray(indices, dtype=np.int64).astype(np.uint64)
    k = np.arange(1, v.shape[0] + 1, dtype=np.uint64)
    s = int(np.sum(k * v, dtype=np.uint64))
    return s - (1 << 64) if s >= 1 << 63 else s


_INDEX_TYPES = {"cubic": 1, "hilbert": 2}   # IDX_CUBIC, IDX_HILBERT (src/grid/index.F90:66-67)


def write_grid_fingerprint(path, mesh: Mesh, index_type: str = "cubic", extent=None) -> None:
    """The restart file "grid" (mesh_write_fingerprint,
    src/grid/mesh.F90:315-352): np_part_global, np_global, algorithm,
    checksum, bits, dim, type, then offset(i) and nn(i) per axis, each a
    20-character label and a 21-wide integer."""
    e = np.asarray(cubic_extent(mesh) if extent is None else extent, dtype=np.int64)
    G = 2 * e + 1
    idx = spatial_index(mesh.lxyz, e, index_type)
    lines = [("np_part_global=", mesh.np_part), ("np_global=", mesh.np), ("algorithm=", 1),
             ("checksum=", index_checksum(idx)), ("bits=", hilbert_bits(e)), ("dim=", 3),
             ("type=", _INDEX_TYPES[index_type])]
    out = [f"{a:<20s}{b:21d}" for a, b in lines]
    # '(a7,i2,a11,i21)': a label shorter than its A field is right-justified
    # ("    nn("), a longer one cut to the field (")=" and 9 blanks)
    out += [f"{'offset(':>7s}{d + 1:2d}{')=':<11s}{int(G[d] // 2):21d}" for d in range(3)]
    out += [f"{'nn(':>7s}{d + 1:2d}{')=':<11s}{int(G[d]):21d}" for d in range(3)]
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def read_grid_fingerprint(path) -> dict:
    """Fields of a restart "grid" file (mesh_read_fingerprint,
    src/grid/mesh.F90:361-446): each line read as a 20-character label and
    an integer."""
    with open(path) as f:
        rows = [ln.rstrip("\n") for ln in f if ln.strip()]
    if len(rows) < 7:
        raise ValueError(f"{path}: fewer than 7 lines")
    val = [int(r[20:41]) for r in rows]
    dim = val[5]
    if len(rows) < 7 + 2 * dim:
        raise ValueError(f"{path}: missing offset or nn lines")
    return {"np_part": val[0], "np": val[1], "algorithm": val[2], "checksum": val[3], "bits": val[4],
            "dim": dim, "type": val[6], "offset": val[7: 7 + dim], "nn": val[7 + dim: 7 + 2 * dim]}


def mesh_from_restart(directory, spacing) -> Mesh:
    """The mesh of a reference restart directory from its "grid" fingerprint
    and indices.obf (what mesh_check_dump_compatibility reads,
    src/grid/mesh.F90:449-533): point order, inner/boundary split and index
    type from the files, the checksum verified; the spacing is an input of
    the run, not stored there."""
    import os
    fp = read_grid_fingerprint(os.path.join(directory, "grid"))
    if fp["dim"] != 3:
        raise ValueError("mesh_from_restart: only 3D meshes")
    types = {v: k for k, v in _INDEX_TYPES.items()}
    if fp["type"] not in types:
        raise ValueError(f"mesh_from_restart: unknown index type {fp['type']}")
    nn = np.asarray(fp["nn"], dtype=np.int64)
    if np.any(nn % 2 == 0) or np.any(np.asarray(fp["offset"]) != nn // 2):
        raise ValueError("mesh_from_restart: only symmetric index ranges (odd nn, offset = nn / 2)")
    idx = read_indices_obf(os.path.join(directory, "indices.obf"))
    if idx.shape[0] != fp["np_part"]:
        raise ValueError("mesh_from_restart: indices.obf and grid disagree on np_part")
    if index_checksum(idx) != fp["checksum"]:
        raise ValueError("mesh_from_restart: index checksum mismatch")
    m = Mesh(lxyz=spatial_point(idx, nn // 2, types[fp["type"]]), np=int(fp["np"]),
             spacing=np.asarray(spacing, dtype=np.float64) * np.ones(3), label=str(directory))
    return m
