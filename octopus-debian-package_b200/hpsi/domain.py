"""Domain-parallel meshes: partitions, ghost rows and their exchange.

The host side of the reference's par_vec_t (src/grid/par_vec.F90:196-420,
par_vec_init) and of X(ghost_update_batch_start/finish)
(src/grid/boundaries_inc.F90:57-231):

* ``partition_z`` splits the inner points of a mesh into ``nparts`` slabs of
  consecutive z planes with about the same number of points (the reference
  takes its partition from METIS or a similar library; a slab partition keeps
  every partition's neighbours to the one below and the one above).
* Each ``Domain`` holds the local mesh of one partition in the par_vec_t row
  order -- its own inner points (in global order), then its ghost points
  grouped by source partition (``ghost_rcounts``/``ghost_rdispls``), then the
  boundary points its stencil reaches -- and the send map: the local rows that
  each other partition holds as ghosts, grouped by destination
  (``ghost_sendmap``, ``ghost_scounts``, ``ghost_sdispls``).
* ``ghost_update`` packs the send rows on the device (``hpsi_ghost_pack``),
  posts one receive and one send per neighbour through ``torch.distributed``
  (NCCL between GPUs) and lands each message in the ghost rows (directly when
  rows are contiguous, through ``hpsi_ghost_unpack`` otherwise).

After the update, H psi of the partition's inner points is ``hpsi_apply_h``
with ``set_bc = 0`` on the local mesh: ghost rows hold the neighbours' values
and boundary rows zeros.  KB spheres may cross partitions: each partition
holds every projector matrix restricted to its own inner points
(``local_projectors``), computes its share of the projections
(``hpsi_projector_bra``), the shares are summed over the partitions (the
mesh%allreduce of X(hamiltonian_elec_base_nlocal_finish),
src/hamiltonian/hamiltonian_elec_base_inc.F90:836) while the stencil pass
runs, and the sum is added back on the partition's covered rows
(``hpsi_projector_ket``): ``apply_partitioned``.

The Taylor exponential on partitions (``taylor_partitioned``) runs its
Horner levels one at a time, each after a ghost update of its input:
``hpsi_apply_h_horner`` for the kinetic and local terms and, with KB spheres,
the summed projections added with the level's factor -i dt / k.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .mesh import Mesh
from .stencil import star_points


@dataclass
class Domain:
    rank: int
    nparts: int
    mesh: Mesh                  # local mesh: inner | ghosts by source | boundary
    global_rows: np.ndarray     # global row of every local row
    np_ghost: int
    ghost_rcounts: np.ndarray   # (nparts,) ghost rows received from each partition
    ghost_rdispls: np.ndarray   # (nparts,) their offsets after the inner rows
    ghost_sendmap: np.ndarray   # local rows sent, grouped by destination
    ghost_scounts: np.ndarray   # (nparts,)
    ghost_sdispls: np.ndarray   # (nparts,)
    _dev: dict = field(default_factory=dict, repr=False)

    @property
    def np_local(self) -> int:
        return self.mesh.np

    @property
    def inner_rows(self) -> np.ndarray:
        """Global rows of this partition's inner points."""
        return self.global_rows[: self.mesh.np]

    def local_batch(self, psi_global: np.ndarray) -> np.ndarray:
        """Local rows of a global (np_part, ld) batch: inner and ghost rows
        copied, boundary rows zero (the zero boundary)."""
        out = np.zeros((self.mesh.np_part,) + psi_global.shape[1:], dtype=psi_global.dtype)
        n = self.mesh.np + self.np_ghost
        out[:n] = psi_global[self.global_rows[:n]]
        return out

    def device_maps(self, device):
        """int32 device copies of the send map and the ghost row positions."""
        import torch
        key = str(device)
        if key not in self._dev:
            ghost_pos = np.arange(self.mesh.np, self.mesh.np + self.np_ghost, dtype=np.int32)
            self._dev[key] = (torch.from_numpy(self.ghost_sendmap.astype(np.int32)).to(device),
                              torch.from_numpy(ghost_pos).to(device))
        return self._dev[key]


def _lookup(lxyz: np.ndarray):
    lo = lxyz.min(0)
    ext = lxyz.max(0) - lo + 1
    lut = -np.ones(int(np.prod(ext)), dtype=np.int64)
    def flat(c):
        c = c - lo
        return (c[..., 2] * ext[1] + c[..., 1]) * ext[0] + c[..., 0]
    lut[flat(lxyz)] = np.arange(len(lxyz))
    def find(c):
        inside = np.all((c >= lo) & (c < lo + ext), axis=-1)
        out = -np.ones(c.shape[:-1], dtype=np.int64)
        out[inside] = lut[flat(c[inside])]
        return out
    return find


def partition_z(mesh: Mesh, nparts: int, order: int = 4) -> list[Domain]:
    """Slab partition of the inner points along z and the ghost layout of
    every partition (par_vec_init, src/grid/par_vec.F90:196-420)."""
    if mesh.periodic:
        raise ValueError("partition_z: periodic meshes are not partitioned here")
    if nparts < 1:
        raise ValueError("partition_z: nparts must be >= 1")
    L = np.asarray(mesh.lxyz, dtype=np.int64)
    npi = mesh.np
    z = L[:npi, 2]
    zs, cnt = np.unique(z, return_counts=True)
    if nparts > len(zs):
        raise ValueError("partition_z: more partitions than z planes")
    # cut after the plane where the cumulative count passes k/nparts of the points
    cum = np.cumsum(cnt)
    cuts, prev = [], -1
    for k in range(1, nparts):
        i = int(np.searchsorted(cum, k * npi / nparts))
        # at least one plane in this partition and in each of the remaining ones
        i = min(max(i, prev + 1), len(zs) - 1 - (nparts - k))
        cuts.append(i)
        prev = i
    zcut = np.array([zs[i] for i in cuts], dtype=np.int64)   # last plane of partitions 0..nparts-2
    part = np.searchsorted(zcut, z, side="left").astype(np.int64)
    find = _lookup(L)
    pts = star_points(order).astype(np.int64)

    inner = [np.nonzero(part == p)[0] for p in range(nparts)]
    needed = []
    for p in range(nparts):
        nb = find(L[inner[p]][:, None, :] + pts[None, :, :]).ravel()
        if (nb < 0).any():
            raise ValueError("partition_z: a stencil neighbour of an inner point is not in the mesh")
        nb = np.unique(nb)
        mine = np.zeros(L.shape[0], dtype=bool)
        mine[inner[p]] = True
        needed.append(nb[~mine[nb]])

    ghosts = [[np.zeros(0, dtype=np.int64)] * nparts for _ in range(nparts)]  # ghosts[p][q]
    bnds = []
    for p in range(nparts):
        nd = needed[p]
        gi = nd[nd < npi]
        for q in range(nparts):
            if q != p:
                ghosts[p][q] = np.sort(gi[part[gi] == q])
        bnds.append(np.sort(nd[nd >= npi]))

    doms = []
    for p in range(nparts):
        rc = np.array([len(ghosts[p][q]) for q in range(nparts)], dtype=np.int64)
        rd = np.concatenate([[0], np.cumsum(rc)[:-1]]).astype(np.int64)
        grow = np.concatenate([inner[p]] + [ghosts[p][q] for q in range(nparts)] + [bnds[p]]).astype(np.int64)
        sc = np.array([len(ghosts[d][p]) for d in range(nparts)], dtype=np.int64)
        sd = np.concatenate([[0], np.cumsum(sc)[:-1]]).astype(np.int64)
        # rows of partition p that partition d holds as ghosts, in d's order,
        # as local rows of p (its inner rows are in ascending global order)
        smap = [np.searchsorted(inner[p], ghosts[d][p]) for d in range(nparts)]
        smap = np.concatenate(smap).astype(np.int64) if smap else np.zeros(0, dtype=np.int64)
        local = Mesh(lxyz=np.ascontiguousarray(L[grow].astype(np.int32)), np=len(inner[p]),
                     spacing=np.asarray(mesh.spacing, dtype=np.float64).copy(),
                     label=f"{mesh.label} part {p}/{nparts}")
        doms.append(Domain(rank=p, nparts=nparts, mesh=local, global_rows=grow, np_ghost=int(rc.sum()),
                           ghost_rcounts=rc, ghost_rdispls=rd, ghost_sendmap=smap,
                           ghost_scounts=sc, ghost_sdispls=sd))
    for p in range(nparts):
        for d in range(nparts):
            assert doms[p].ghost_scounts[d] == doms[d].ghost_rcounts[p]
    return doms


def ghost_update(dom: Domain, psi, nst=None, group=None, pack=None, unpack=None, sendbuf=None, recvbuf=None):
    """Fill the ghost rows of the local batch ``psi`` (npts, ld) from the
    neighbouring partitions; every rank of ``group`` calls it together.

    ``pack(psi, sendmap, out, nst)`` and ``unpack(buf, pos, psi, nst)`` default
    to the device kernels (hpsi_ghost_pack / hpsi_ghost_unpack); ``sendbuf`` and
    ``recvbuf`` may pass preallocated (rows, nst) buffers.  Receives are posted
    for every partition with ghost rows here, sends for every partition that
    holds rows of this one, all at once (torch.distributed.batch_isend_irecv,
    the reference's ring of irecv/isend), then waited for."""
    ghost_update_finish(ghost_update_start(dom, psi, nst=nst, group=group, pack=pack, unpack=unpack,
                                           sendbuf=sendbuf, recvbuf=recvbuf))


def ghost_update_start(dom: Domain, psi, nst=None, group=None, pack=None, unpack=None, sendbuf=None, recvbuf=None):
    """Post the ghost exchange of ``psi`` (X(ghost_update_batch_start),
    src/grid/boundaries_inc.F90:57-148) and return its handle for
    ``ghost_update_finish``; the ghost rows of ``psi`` are undefined until
    then.  Every rank of ``group`` calls it together."""
    import torch
    import torch.distributed as dist
    from . import lib
    pack = pack or lib.ghost_pack
    unpack = unpack or lib.ghost_unpack
    nst = psi.shape[1] if nst is None else nst
    ld = psi.shape[1]
    dev = psi.device
    nsend = int(dom.ghost_scounts.sum())
    sendmap, ghost_pos = dom.device_maps(dev)
    if sendbuf is None:
        sendbuf = torch.empty((nsend, nst), dtype=psi.dtype, device=dev)
    if nsend:
        pack(psi, sendmap, sendbuf, nst=nst)
        # NCCL orders its sends after the work already queued on the current
        # stream (the pack); other backends read the buffer from the host side
        if dev.type == "cuda" and dist.get_backend(group) != "nccl":
            torch.cuda.current_stream(dev).synchronize()
    direct = ld == nst
    if not direct and recvbuf is None:
        recvbuf = torch.empty((dom.np_ghost, nst), dtype=psi.dtype, device=dev)
    ops = []
    # receives first, counting upwards from this rank (the reference's ring order)
    for k in range(dom.nparts):
        q = (dom.rank + k) % dom.nparts
        n = int(dom.ghost_rcounts[q])
        if q == dom.rank or n == 0:
            continue
        off = int(dom.ghost_rdispls[q])
        tgt = psi[dom.np_local + off: dom.np_local + off + n] if direct else recvbuf[off: off + n]
        ops.append(dist.P2POp(dist.irecv, torch.view_as_real(tgt), q, group=group))
    for k in range(dom.nparts):
        q = (dom.rank - k) % dom.nparts
        n = int(dom.ghost_scounts[q])
        if q == dom.rank or n == 0:
            continue
        off = int(dom.ghost_sdispls[q])
        ops.append(dist.P2POp(dist.isend, torch.view_as_real(sendbuf[off: off + n]), q, group=group))
    reqs = dist.batch_isend_irecv(ops) if ops else []
    return {"reqs": reqs, "dom": dom, "psi": psi, "nst": nst, "direct": direct, "recvbuf": recvbuf,
            "ghost_pos": ghost_pos, "unpack": unpack, "sendbuf": sendbuf}


def ghost_update_finish(handle):
    """Wait for the exchange ``ghost_update_start`` posted and land the
    messages in the ghost rows (X(ghost_update_batch_finish),
    src/grid/boundaries_inc.F90:150-231)."""
    for r in handle["reqs"]:
        r.wait()
    dom = handle["dom"]
    if not handle["direct"] and dom.np_ghost:
        handle["unpack"](handle["recvbuf"], handle["ghost_pos"], handle["psi"], nst=handle["nst"])


def local_projectors(dom: Domain, projectors):
    """Every projector matrix restricted to the partition's inner points:
    the sphere points this partition owns, as local rows, with their rows of
    the matrix; a matrix with no point here keeps its projectors (and zero
    points), so the projection rows of all partitions line up for the sum
    (the reference builds the projector maps from the local points of each
    domain, src/hamiltonian/hamiltonian_elec_base.F90:715-718)."""
    from .fixtures import ProjectorSet
    nglob = int(dom.global_rows.max()) + 1 if dom.global_rows.size else 0
    nglob = max(nglob, max((int(np.max(m)) + 1 for m in projectors.maps if len(m)), default=0))
    loc = -np.ones(nglob, dtype=np.int64)
    loc[dom.inner_rows] = np.arange(dom.np_local)
    maps, mats = [], []
    for mp, mt in zip(projectors.maps, projectors.mats):
        mp = np.asarray(mp, dtype=np.int64)
        li = loc[mp]
        sel = li >= 0
        maps.append(li[sel].astype(np.int32))
        mats.append(np.ascontiguousarray(np.asarray(mt, dtype=np.float64)[sel]))
    return ProjectorSet(maps, mats, [np.asarray(c, dtype=np.float64) for c in projectors.scals],
                        getattr(projectors, "positions", None))


def local_projector_phases(dom: Domain, projectors, phases):
    """The projector phases (k != 0, one complex number per sphere point of
    each matrix, src/hamiltonian/projector.F90:171-247) restricted with the
    same point selection as ``local_projectors``: the phases of this
    partition's own sphere points, in the order of its local maps."""
    nglob = int(dom.global_rows.max()) + 1 if dom.global_rows.size else 0
    nglob = max(nglob, max((int(np.max(m)) + 1 for m in projectors.maps if len(m)), default=0))
    loc = -np.ones(nglob, dtype=np.int64)
    loc[dom.inner_rows] = np.arange(dom.np_local)
    out = []
    for mp, ph in zip(projectors.maps, phases):
        ph = np.asarray(ph, dtype=np.complex128)
        if len(ph) != len(mp):
            raise ValueError("local_projector_phases: one phase per sphere point of each matrix expected")
        out.append(np.ascontiguousarray(ph[loc[np.asarray(mp, dtype=np.int64)] >= 0]))
    return out


POINTS_ALL, POINTS_INNER, POINTS_OUTER = 0, 1, 2


def apply_partitioned(dom: Domain, psi, hpsi, local_apply, bra=None, ket=None, proj=None, nst=None, group=None,
                      pack=None, unpack=None, overlap=False):
    """H psi of one partition; every rank of ``group`` calls it together.

    1. ghost update of ``psi`` (``ghost_update``);
    2. if ``bra`` is given: ``bra(psi, proj)`` writes this partition's share of
       the KB projections into ``proj`` (nprojections, ld) and an
       asynchronous all-reduce sums the shares over the ranks
       (X(hamiltonian_elec_base_nlocal_start) and the mesh%allreduce of
       hamiltonian_elec_base_inc.F90:836);
    3. ``local_apply(psi, hpsi, points)``: kinetic and local terms on the local
       mesh, overlapping the all-reduce;
    4. wait for the sum, then ``ket(proj, hpsi)`` adds the KB term on the
       covered rows (X(hamiltonian_elec_base_nlocal_finish)).
    With ``overlap`` the ghost exchange is only posted in step 1 and the bra
    (which reads this partition's own points only) and the pass over the
    points whose stencil reads no ghost row (``points = POINTS_INNER``) run
    while the messages are in flight; the exchange is then finished and the
    other points follow (``POINTS_OUTER``), as X(derivatives_batch_start/
    finish) overlap them (src/grid/derivatives_inc.F90:82-102).  Without it
    ``local_apply`` gets ``POINTS_ALL``.  With NCCL the all-reduce runs on its
    own stream after the bra and the ket's stream waits for it; nothing
    synchronises the host."""
    import torch
    import torch.distributed as dist
    handle = ghost_update_start(dom, psi, nst=nst, group=group, pack=pack, unpack=unpack)
    if not overlap:
        ghost_update_finish(handle)
    work = None
    if bra is not None:
        bra(psi, proj)
        if dom.nparts > 1:
            work = dist.all_reduce(torch.view_as_real(proj), group=group, async_op=True)
    if overlap:
        local_apply(psi, hpsi, POINTS_INNER)
        ghost_update_finish(handle)
        local_apply(psi, hpsi, POINTS_OUTER)
    else:
        local_apply(psi, hpsi, POINTS_ALL)
    if bra is not None:
        if work is not None:
            work.wait()
        ket(proj, hpsi)


def taylor_partitioned(dom: Domain, psi, work, horner, bra=None, ket=None, proj=None, dt=0.0, order=4, nst=None,
                       group=None, pack=None, unpack=None, overlap=False):
    """psi <- sum_{k=0..order} (-i dt H)^k / k! psi on this partition's inner
    rows, every rank of ``group`` calling it together: the Taylor series of
    exponential_taylor_series_batch (src/electrons/exponential.F90:677-757)
    in Horner form, in <- psi + (-i dt / k) H in for k = order..1, each level
    after a ghost update of its input (X(ghost_update_batch_start/finish)
    inside every H psi of the reference's domain-parallel run).

    ``work`` holds two (npts, ld) batches like ``psi`` whose boundary rows are
    zero; ``horner(x, psi0, out, a, points)`` writes out = psi0 + a (T + V) x
    on the points of ``points`` (hpsi_apply_h_horner_points, set_bc = 0);
    with KB projectors ``bra(x, proj)`` writes this partition's projection
    share, summed over the ranks while the pass runs, and ``ket(proj, out, a)``
    adds a P proj.  ``overlap`` runs the inner points of each level while its
    ghost rows are in flight, as ``apply_partitioned`` does."""
    import torch
    import torch.distributed as dist
    if order < 1:
        raise ValueError("taylor_partitioned: order must be >= 1")
    dt = complex(dt)
    x = psi
    for k in range(order, 0, -1):
        a = -1j * dt / k
        out = work[(order - k) % 2] if (k > 1 or order == 1) else psi
        handle = ghost_update_start(dom, x, nst=nst, group=group, pack=pack, unpack=unpack)
        if not overlap:
            ghost_update_finish(handle)
        work_ar = None
        if bra is not None:
            bra(x, proj)
            if dom.nparts > 1:
                work_ar = dist.all_reduce(torch.view_as_real(proj), group=group, async_op=True)
        if overlap:
            horner(x, psi, out, a, POINTS_INNER)
            ghost_update_finish(handle)
            horner(x, psi, out, a, POINTS_OUTER)
        else:
            horner(x, psi, out, a, POINTS_ALL)
        if bra is not None:
            if work_ar is not None:
                work_ar.wait()
            ket(proj, out, a)
        x = out
    if order == 1:
        psi[: dom.np_local].copy_(x[: dom.np_local])


class DomainHamiltonian:
    """H psi of one partition on its local mesh: kinetic, local and KB terms
    (KB spheres may cross partitions)."""

    def __init__(self, dom: Domain, weights, points, v_global=None, projectors=None, projector_phases=None):
        """``projector_phases``: the global phases (one array per matrix, in
        the global maps' order) for k != 0; each partition keeps those of
        its own sphere points."""
        from . import lib
        self.dom = dom
        self.dmesh = lib.DeviceMesh(dom.mesh)
        v = None if v_global is None else np.asarray(v_global)[dom.inner_rows]
        self.local_proj = None if projectors is None else local_projectors(dom, projectors)
        self.ham = lib.Hamiltonian(self.dmesh, weights, points, v=v, projectors=self.local_proj)
        # the ghost rows follow the partition's own points (par_vec_t order)
        self.dmesh.set_ghost_rows(dom.np_local, dom.np_ghost)
        if projector_phases is not None:
            if projectors is None:
                raise ValueError("DomainHamiltonian: projector phases without projectors")
            self.ham.set_projector_phases(local_projector_phases(dom, projectors, projector_phases))
        self.nprojections = self.ham.nprojections()
        self._proj = {}

    def projection_buffer(self, psi):
        """The (nprojections, ld) device buffer of the summed projections for
        batches like ``psi`` (kept between calls)."""
        import torch
        key = (psi.dtype, psi.shape[1], str(psi.device))
        if key not in self._proj:
            self._proj[key] = torch.zeros((self.nprojections, psi.shape[1]), dtype=psi.dtype, device=psi.device)
        return self._proj[key]

    def apply(self, psi, hpsi, nst=None, group=None, overlap=True):
        """Ghost update of ``psi`` (boundary rows must be zero), then H psi of
        the inner rows into ``hpsi``: hpsi_apply_h_points (set_bc = 0) for the
        kinetic and local terms, the points that read no ghost row while the
        ghost rows are in flight (``overlap``), the projections summed over
        the ranks of ``group`` and the KB ket (``apply_partitioned``)."""
        from . import lib
        kb = self.nprojections > 0
        terms = lib.TERM_KINETIC | lib.TERM_LOCAL_POTENTIAL
        apply_partitioned(
            self.dom, psi, hpsi,
            lambda x, y, pts: self.ham.apply(x, y, nst=nst, terms=terms, set_bc=False, points=pts),
            bra=self.ham.projector_bra if kb else None,
            ket=(lambda p, y: self.ham.projector_ket(p, y, nst=nst)) if kb else None,
            proj=self.projection_buffer(psi) if kb else None, nst=nst, group=group, overlap=overlap)

    def taylor_step(self, psi, dt, order=4, nst=None, group=None, overlap=True):
        """psi <- exp(-i dt H) psi (order-``order`` Taylor) on the partition's
        inner rows; ``psi`` is the local (np_part, ld) device batch with zero
        boundary rows (``taylor_partitioned``)."""
        import torch
        from . import lib
        key = ("work", psi.dtype, psi.shape, str(psi.device))
        if key not in self._proj:
            self._proj[key] = [torch.zeros_like(psi), torch.zeros_like(psi)]
        kb = self.nprojections > 0
        terms = lib.TERM_KINETIC | lib.TERM_LOCAL_POTENTIAL
        taylor_partitioned(
            self.dom, psi, self._proj[key],
            lambda x, p0, y, a, pts: self.ham.apply_horner(x, p0, y, a, nst=nst, terms=terms, set_bc=False,
                                                           points=pts),
            bra=self.ham.projector_bra if kb else None,
            ket=(lambda p, y, a: self.ham.projector_ket(p, y, nst=nst, a=a)) if kb else None,
            proj=self.projection_buffer(psi) if kb else None, dt=dt, order=order, nst=nst, group=group,
            overlap=overlap)
