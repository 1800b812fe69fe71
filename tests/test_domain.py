"""Domain-parallel meshes on the CPU: partition layout, the oracle's ghost
exchange, H psi of the partitions against the global H psi, and the
torch.distributed exchange protocol over gloo with two ranks."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import small_sphere_system

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("nparts", [1, 2, 3, 5])
def test_partition_layout_and_partitioned_hpsi(nparts):
    from hpsi.domain import partition_z
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O
    m, v, proj, psi = small_sphere_system(seed=11, nst=3)
    doms = partition_z(m, nparts)
    inner = np.concatenate([d.inner_rows for d in doms])
    assert np.array_equal(np.sort(inner), np.arange(m.np))
    w = laplacian_weights(m.spacing)
    Hg = O.Hamiltonian(m, w, star_points(), v=v)
    ref = Hg.apply(psi)
    # local batches with the ghost rows still empty, then the oracle exchange
    locs = []
    for d in doms:
        b = d.local_batch(psi)
        b[d.np_local: d.np_local + d.np_ghost] = 0.0
        locs.append(b)
    O.ghost_exchange(doms, locs)
    for d, b in zip(doms, locs):
        n = d.np_local + d.np_ghost
        assert np.array_equal(b[:n], psi[d.global_rows[:n]])
        assert not b[n:].any()
        H = O.Hamiltonian(d.mesh, w, star_points(), v=v[d.inner_rows], bc="none")
        got = H.apply(b)
        assert np.max(np.abs(got - ref[d.inner_rows])) <= 1e-13 * np.max(np.abs(ref))
    for p, d in enumerate(doms):
        assert d.ghost_rcounts[p] == 0 and d.ghost_scounts[p] == 0
        if nparts > 1:
            assert d.np_ghost > 0
        else:
            assert d.np_ghost == 0 and d.ghost_sendmap.size == 0 and d.mesh.np == m.np


def test_partition_rejects_periodic_and_too_many_parts():
    from hpsi.domain import partition_z
    from hpsi.mesh import index_box_mesh
    m = index_box_mesh((6, 5, 4), 0.3)
    with pytest.raises(ValueError):
        partition_z(m, 5)
    m.periodic = True
    with pytest.raises(ValueError):
        partition_z(m, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "octopus-debian-package_b200"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from helpers import small_sphere_system
    from hpsi.domain import ghost_update, partition_z

    # CPU stand-ins for the device pack/unpack kernels (the test checks the
    # exchange protocol: counts, offsets, ring order, direct and buffered receives)
    def pack(psi, sendmap, out, nst):
        out.copy_(psi[sendmap.long(), :nst])

    def unpack(buf, pos, psi, nst):
        psi[pos.long(), :nst] = buf

    m, v, proj, psi = small_sphere_system(seed=13, nst=4)
    d = partition_z(m, world)[rank]
    ok = []
    for ld in (4, 8):
        g = np.zeros((m.np_part, ld), dtype=np.complex128)
        g[:, :4] = psi
        b = d.local_batch(g)
        b[d.np_local: d.np_local + d.np_ghost] = 0.0
        t = torch.from_numpy(b)
        ghost_update(d, t, nst=4, pack=pack, unpack=unpack)
        n = d.np_local + d.np_ghost
        ok.append(bool(np.array_equal(t.numpy()[:n], g[d.global_rows[:n]])))
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, ok))


def test_ghost_update_gloo_two_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: [True, True], 1: [True, True]}


@pytest.mark.parametrize("nparts", [2, 3, 5])
def test_partitioned_hpsi_with_kb_spheres_across_partitions(nparts):
    """Each partition's share of the KB projections (its own sphere points
    only), summed over the partitions, then added back on its covered rows:
    the partitioned H psi with every term equals the global one."""
    from hpsi.domain import local_projectors, partition_z
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O
    m, v, proj, psi = small_sphere_system(seed=19, nst=3, natoms=4)
    w = laplacian_weights(m.spacing)
    ref = O.Hamiltonian(m, w, star_points(), v=v,
                        projectors=O.Projectors(proj.maps, proj.mats, proj.scals)).apply(psi)
    doms = partition_z(m, nparts)
    locs = [d.local_batch(psi) for d in doms]
    O.ghost_exchange(doms, locs)
    lps = [local_projectors(d, proj) for d in doms]
    # at least one sphere is split between partitions
    split = [sum(len(lp.maps[i]) > 0 for lp in lps) for i in range(len(proj.maps))]
    assert max(split) > 1
    for lp, d in zip(lps, doms):
        assert sum(len(a) for a in lp.maps) <= d.np_local
    total = sum(O.kb_bra(lp.maps, lp.mats, lp.scals, b[: d.np_local]) for lp, d, b in zip(lps, doms, locs))
    full = O.kb_bra(proj.maps, proj.mats, proj.scals, psi)
    assert np.max(np.abs(total - full)) <= 1e-13 * np.max(np.abs(full))
    for lp, d, b in zip(lps, doms, locs):
        h = O.Hamiltonian(d.mesh, w, star_points(), v=v[d.inner_rows], bc="none").apply(b)
        O.kb_ket(lp.maps, lp.mats, total, h)
        assert np.max(np.abs(h - ref[d.inner_rows])) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("nparts", [2, 3])
def test_partitioned_kb_with_projector_phases(nparts):
    """k != 0: each partition keeps the phases of its own sphere points
    (local_projector_phases, the selection of local_projectors); the summed
    shares and the ket on every partition equal the global KB term with
    phases."""
    from hpsi.domain import local_projector_phases, local_projectors, partition_z
    from oracle import oracle as O
    m, v, proj, psi = small_sphere_system(seed=23, nst=3, natoms=4)
    rng = np.random.default_rng(24)
    ph = [np.exp(1j * rng.uniform(0, 2 * np.pi, len(mp))) for mp in proj.maps]
    full = O.kb_bra(proj.maps, proj.mats, proj.scals, psi, ph)
    ref = O.kb_ket(proj.maps, proj.mats, full, np.zeros((m.np, 3), complex), ph)
    doms = partition_z(m, nparts)
    locs = [d.local_batch(psi) for d in doms]
    lps = [local_projectors(d, proj) for d in doms]
    lph = [local_projector_phases(d, proj, ph) for d in doms]
    for lp, p_ in zip(lps, lph):
        assert [len(a) for a in lp.maps] == [len(a) for a in p_]
    total = sum(O.kb_bra(lp.maps, lp.mats, lp.scals, b[: d.np_local], p_)
                for lp, p_, d, b in zip(lps, lph, doms, locs))
    assert np.max(np.abs(total - full)) <= 1e-13 * np.max(np.abs(full))
    for lp, p_, d in zip(lps, lph, doms):
        h = O.kb_ket(lp.maps, lp.mats, total, np.zeros((d.np_local, 3), complex), p_)
        assert np.max(np.abs(h - ref[d.inner_rows])) <= 1e-13 * np.max(np.abs(ref))
    with pytest.raises(ValueError):
        local_projector_phases(doms[0], proj, [p_[:-1] for p_ in ph])


def _rank_kb_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "octopus-debian-package_b200"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from helpers import small_sphere_system
    from hpsi.domain import apply_partitioned, local_projectors, partition_z
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O

    # CPU stand-ins for the device kernels: the test checks the protocol
    # (ghost exchange, projection shares summed by the all-reduce, ket after it)
    def pack(psi, sendmap, o, nst):
        o.copy_(psi[sendmap.long(), :nst])

    def unpack(buf, pos, psi, nst):
        psi[pos.long(), :nst] = buf

    m, v, proj, psi = small_sphere_system(seed=19, nst=3, natoms=4)
    w = laplacian_weights(m.spacing)
    ref = O.Hamiltonian(m, w, star_points(), v=v,
                        projectors=O.Projectors(proj.maps, proj.mats, proj.scals)).apply(psi)
    d = partition_z(m, world)[rank]
    lp = local_projectors(d, proj)
    Hl = O.Hamiltonian(d.mesh, w, star_points(), v=v[d.inner_rows], bc="none")
    b = d.local_batch(psi)
    b[d.np_local: d.np_local + d.np_ghost] = 0.0
    pr = torch.zeros((sum(mt.shape[1] for mt in lp.mats), 3), dtype=torch.complex128)
    # the partition's points whose star reads no ghost row; the inner part
    # runs on a copy whose ghost rows are NaN, so reading one would show
    ghost = np.zeros(d.mesh.np_part, dtype=bool)
    ghost[d.np_local: d.np_local + d.np_ghost] = True
    clean = ~ghost[O.neighbour_table(d.mesh, star_points())].any(axis=1)

    def part_rows(pts):
        return slice(None) if pts == 0 else (clean if pts == 1 else ~clean)

    def local_in(a, pts):
        an = a.numpy()
        if pts == 1:
            an = an.copy()
            an[ghost] = np.nan
        return an

    def bra(a, p):
        p.copy_(torch.from_numpy(O.kb_bra(lp.maps, lp.mats, lp.scals, a.numpy()[: d.np_local])))

    def ket(p, h):
        hn = h.numpy()
        O.kb_ket(lp.maps, lp.mats, p.numpy(), hn)

    def local_apply(a, h, pts):
        r = Hl.apply(local_in(a, pts))
        h.numpy()[part_rows(pts)] = r[part_rows(pts)]

    errs = []
    for overlap in (False, True):
        x = torch.from_numpy(b.copy())
        y = torch.zeros((d.np_local, 3), dtype=torch.complex128)
        apply_partitioned(d, x, y, local_apply, bra=bra, ket=ket, proj=pr, pack=pack, unpack=unpack,
                          overlap=overlap)
        errs.append(float(np.max(np.abs(y.numpy() - ref[d.inner_rows])) / np.max(np.abs(ref))))
    err = max(errs)

    # Taylor step level by level (ghost update and projection sum per level)
    from hpsi.domain import taylor_partitioned
    dt = 0.02
    ref_t = O.Hamiltonian(m, w, star_points(), v=v,
                          projectors=O.Projectors(proj.maps, proj.mats, proj.scals)).taylor(psi, dt)

    def horner(a_in, p0, o, a, pts):
        r = p0.numpy()[: d.np_local] + a * Hl.apply(local_in(a_in, pts))
        o.numpy()[: d.np_local][part_rows(pts)] = r[part_rows(pts)]

    def ket_a(p, h, a):
        hn = h.numpy()
        hn[: d.np_local] += a * O.kb_ket(lp.maps, lp.mats, p.numpy(), np.zeros((d.np_local, 3), complex))

    errs_t = []
    for overlap in (False, True):
        x = torch.from_numpy(b.copy())
        x[d.np_local: d.np_local + d.np_ghost] = 0.0
        work = [torch.zeros_like(x), torch.zeros_like(x)]
        taylor_partitioned(d, x, work, horner, bra=bra, ket=ket_a, proj=pr, dt=dt, order=4, pack=pack,
                           unpack=unpack, overlap=overlap)
        errs_t.append(float(np.max(np.abs(x.numpy()[: d.np_local] - ref_t[d.inner_rows])) / np.max(np.abs(ref_t))))
    err_t = max(errs_t)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, (err, err_t)))


def test_partitioned_kb_gloo_two_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_kb_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert set(res) == {0, 1}
    assert max(e for e, _ in res.values()) <= 1e-13
    assert max(t for _, t in res.values()) <= 1e-12


@pytest.mark.parametrize("order", [1, 2, 4])
def test_taylor_partitioned_single_partition_orders(order):
    """One partition (no exchange, no all-reduce): the level-by-level Taylor
    step with oracle stand-ins equals the oracle's Taylor step of each order,
    order 1 included (its result lands in a work batch and is copied back)."""
    import torch
    from hpsi.domain import local_projectors, partition_z, taylor_partitioned
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O
    m, v, proj, psi = small_sphere_system(seed=43, nst=2, natoms=2)
    w = laplacian_weights(m.spacing)
    dt = 0.03
    ref = O.Hamiltonian(m, w, star_points(), v=v,
                        projectors=O.Projectors(proj.maps, proj.mats, proj.scals)).taylor(psi, dt, order=order)
    d = partition_z(m, 1)[0]
    lp = local_projectors(d, proj)
    Hl = O.Hamiltonian(d.mesh, w, star_points(), v=v[d.inner_rows], bc="none")
    x = torch.from_numpy(d.local_batch(psi))
    work = [torch.zeros_like(x), torch.zeros_like(x)]
    pr = torch.zeros((sum(mt.shape[1] for mt in lp.mats), 2), dtype=torch.complex128)

    def horner(a_in, p0, o, a, pts):
        assert pts == 0
        o[: d.np_local] = p0[: d.np_local] + a * torch.from_numpy(Hl.apply(a_in.numpy()))

    def bra(a_in, p):
        p.copy_(torch.from_numpy(O.kb_bra(lp.maps, lp.mats, lp.scals, a_in.numpy()[: d.np_local])))

    def ket(p, h, a):
        h.numpy()[: d.np_local] += a * O.kb_ket(lp.maps, lp.mats, p.numpy(), np.zeros((d.np_local, 2), complex))

    taylor_partitioned(d, x, work, horner, bra=bra, ket=ket, proj=pr, dt=dt, order=order)
    got = x.numpy()[: d.np_local]
    assert np.max(np.abs(got - ref[d.inner_rows])) <= 1e-12 * np.max(np.abs(ref))


def test_local_projectors_partition_without_spheres():
    """A partition that no sphere reaches keeps every matrix with zero
    points: its projection share is zero and its rows still line up."""
    from hpsi.domain import local_projectors, partition_z
    from oracle import oracle as O
    m, v, proj, psi = small_sphere_system(seed=47, nst=2, natoms=1)
    doms = partition_z(m, 5)
    lps = [local_projectors(d, proj) for d in doms]
    empty = [i for i, lp in enumerate(lps) if all(len(a) == 0 for a in lp.maps)]
    assert empty, "expected a partition outside the one sphere"
    lp, d = lps[empty[0]], doms[empty[0]]
    assert [mt.shape[1] for mt in lp.mats] == [mt.shape[1] for mt in proj.mats]
    share = O.kb_bra(lp.maps, lp.mats, lp.scals, d.local_batch(psi)[: d.np_local])
    assert share.shape == (sum(mt.shape[1] for mt in proj.mats), 2) and not share.any()
