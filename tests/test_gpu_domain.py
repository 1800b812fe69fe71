"""Domain-parallel H psi on one GPU: the partitions run one after another in
this process, their ghost rows packed by hpsi_ghost_pack and delivered by
device copies (the part NCCL does between GPUs) or hpsi_ghost_unpack; the
partitions' H psi must equal the global H psi of the same states, and the
assembled partitioned result is also checked against the FP64 CPU oracle at
the parity tolerances (FP64 1e-12, FP32 storage 2e-5, relative max-norm per
state)."""
import numpy as np
import pytest

from helpers import rel_maxnorm_per_state, small_sphere_system


def _oracle(m, w, v, proj=None):
    from hpsi.stencil import star_points
    from oracle import oracle as O
    P = O.Projectors(proj.maps, proj.mats, proj.scals) if proj is not None else None
    return O.Hamiltonian(m, w, star_points(), v=v, projectors=P)

pytestmark = pytest.mark.gpu


def _exchange_on_one_gpu(doms, locs, nst):
    import torch
    from hpsi import lib
    sends = []
    for d, b in zip(doms, locs):
        smap, _ = d.device_maps(b.device)
        buf = torch.empty((int(d.ghost_scounts.sum()), nst), dtype=b.dtype, device=b.device)
        if buf.shape[0]:
            lib.ghost_pack(b, smap, buf, nst=nst)
        sends.append(buf)
    for p, d in enumerate(doms):
        ld = locs[p].shape[1]
        recv = torch.empty((d.np_ghost, nst), dtype=locs[p].dtype, device=locs[p].device)
        for q, dq in enumerate(doms):
            n = int(d.ghost_rcounts[q])
            if n == 0:
                continue
            so, ro = int(dq.ghost_sdispls[p]), int(d.ghost_rdispls[q])
            if ld == nst:  # contiguous rows: the message lands in the ghost rows
                locs[p][d.np_local + ro: d.np_local + ro + n].copy_(sends[q][so: so + n])
            else:
                recv[ro: ro + n].copy_(sends[q][so: so + n])
        if ld != nst and d.np_ghost:
            _, pos = d.device_maps(locs[p].device)
            lib.ghost_unpack(recv, pos, locs[p], nst=nst)


@pytest.mark.parametrize("nparts,ld,dtype", [(2, 16, "c128"), (3, 16, "c128"), (3, 24, "c128"), (4, 32, "c64")])
def test_partitioned_hpsi_equals_global(cuda, nparts, ld, dtype):
    import torch
    from hpsi import lib
    from hpsi.domain import DomainHamiltonian, partition_z
    from hpsi.stencil import laplacian_weights, star_points
    nst = 16 if dtype == "c128" else 32
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    m, v, proj, psi = small_sphere_system(seed=17, nst=nst, radius=4.5)
    g = np.zeros((m.np_part, ld), dtype=np.complex128)
    g[:, :nst] = psi
    g[m.np:] = 0.0
    w = laplacian_weights(m.spacing)
    dm = lib.DeviceMesh(m)
    H = lib.Hamiltonian(dm, w, star_points(), v=v)
    x = torch.from_numpy(g).to(cuda).to(tdt)
    y = torch.zeros((m.np, ld), dtype=tdt, device=cuda)
    H.apply(x, y, nst=nst)
    ref = y.cpu().numpy()[:, :nst]
    doms = partition_z(m, nparts)
    hams = [DomainHamiltonian(d, w, star_points(), v_global=v) for d in doms]
    locs = []
    for d in doms:
        b = d.local_batch(g)
        b[d.np_local: d.np_local + d.np_ghost] = 0.0  # filled by the exchange
        locs.append(torch.from_numpy(b).to(cuda).to(tdt))
    _exchange_on_one_gpu(doms, locs, nst)
    tol = 1e-13 if dtype == "c128" else 2e-6
    full = np.zeros((m.np, nst), dtype=np.complex128)
    for d, hm, b in zip(doms, hams, locs):
        n = d.np_local + d.np_ghost
        assert np.array_equal(b.cpu().numpy()[:n, :nst], g[d.global_rows[:n], :nst].astype(b.cpu().numpy().dtype))
        out = torch.zeros((d.np_local, ld), dtype=tdt, device=cuda)
        hm.ham.apply(b, out, nst=nst, set_bc=False)
        got = out.cpu().numpy()[:, :nst]
        assert np.max(np.abs(got - ref[d.inner_rows])) <= tol * np.max(np.abs(ref))
        full[d.inner_rows] = got
    assert rel_maxnorm_per_state(full, _oracle(m, w, v).apply(psi)) <= (1e-12 if dtype == "c128" else 2e-5)


def test_ghost_pack_rejects_host_buffers(cuda):
    import torch
    from hpsi import lib
    x = torch.zeros((10, 4), dtype=torch.complex128, device=cuda)
    smap = torch.arange(3, dtype=torch.int32)
    out = torch.zeros((3, 4), dtype=torch.complex128)
    with pytest.raises(lib.HpsiError):
        lib.ghost_pack(x, smap, out)


def test_ghost_pack_empty_map_is_a_no_op(cuda):
    import torch
    from hpsi import lib
    x = torch.ones((10, 4), dtype=torch.complex64, device=cuda)
    lib.ghost_pack(x, torch.zeros(0, dtype=torch.int32, device=cuda),
                   torch.zeros((0, 4), dtype=torch.complex64, device=cuda))
    lib.ghost_unpack(torch.zeros((0, 4), dtype=torch.complex64, device=cuda),
                     torch.zeros(0, dtype=torch.int32, device=cuda), x)
    assert x.abs().min().item() == 1.0


@pytest.mark.parametrize("dtype,ld,nst", [("c128", 16, 13), ("c64", 32, 32)])
def test_split_kb_term_equals_full_apply(cuda, dtype, ld, nst):
    """hpsi_apply_h without the KB term, then hpsi_projector_bra and
    hpsi_projector_ket, equals hpsi_apply_h with every term."""
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    m, v, proj, psi = small_sphere_system(seed=23, nst=nst, radius=4.5, natoms=4)
    g = np.zeros((m.np_part, ld), dtype=np.complex128)
    g[:, :nst] = psi
    H = lib.Hamiltonian(lib.DeviceMesh(m), laplacian_weights(m.spacing), star_points(), v=v, projectors=proj)
    x = torch.from_numpy(g).to(cuda).to(tdt)
    full = torch.zeros((m.np, ld), dtype=tdt, device=cuda)
    H.apply(x, full, nst=nst)
    part = torch.zeros((m.np, ld), dtype=tdt, device=cuda)
    H.apply(x, part, nst=nst, terms=lib.TERM_KINETIC | lib.TERM_LOCAL_POTENTIAL)
    pr = torch.zeros((H.nprojections(), ld), dtype=tdt, device=cuda)
    assert pr.shape[0] == sum(mt.shape[1] for mt in proj.mats)
    H.projector_bra(x, pr)
    H.projector_ket(pr, part, nst=nst)
    a, b = full.cpu().numpy()[:, :nst], part.cpu().numpy()[:, :nst]
    tol = 1e-13 if dtype == "c128" else 2e-6
    assert np.max(np.abs(a - b)) <= tol * np.max(np.abs(a))


@pytest.mark.parametrize("nparts,ld,dtype", [(2, 16, "c128"), (3, 16, "c128"), (3, 32, "c64")])
def test_partitioned_hpsi_with_kb_equals_global(cuda, nparts, ld, dtype):
    """KB spheres across partitions: each partition's projection share
    (hpsi_projector_bra on its own sphere points), summed on the device (the
    all-reduce NCCL does between GPUs), added back by hpsi_projector_ket after
    the kinetic and local pass; equals the global H psi with every term."""
    import torch
    from hpsi import lib
    from hpsi.domain import DomainHamiltonian, partition_z
    from hpsi.stencil import laplacian_weights, star_points
    nst = 16
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    m, v, proj, psi = small_sphere_system(seed=29, nst=nst, radius=4.5, natoms=4)
    g = np.zeros((m.np_part, ld), dtype=np.complex128)
    g[:, :nst] = psi
    w = laplacian_weights(m.spacing)
    H = lib.Hamiltonian(lib.DeviceMesh(m), w, star_points(), v=v, projectors=proj)
    x = torch.from_numpy(g).to(cuda).to(tdt)
    y = torch.zeros((m.np, ld), dtype=tdt, device=cuda)
    H.apply(x, y, nst=nst)
    ref = y.cpu().numpy()[:, :nst]
    doms = partition_z(m, nparts)
    hams = [DomainHamiltonian(d, w, star_points(), v_global=v, projectors=proj) for d in doms]
    locs = []
    for d in doms:
        b = d.local_batch(g)
        b[d.np_local: d.np_local + d.np_ghost] = 0.0
        locs.append(torch.from_numpy(b).to(cuda).to(tdt))
    _exchange_on_one_gpu(doms, locs, nst)
    shares = []
    for hm, b in zip(hams, locs):
        pr = torch.zeros((hm.nprojections, ld), dtype=tdt, device=cuda)
        hm.ham.projector_bra(b, pr)
        shares.append(pr)
    total = torch.stack(shares).sum(0)
    tol = 1e-13 if dtype == "c128" else 2e-6
    full = np.zeros((m.np, nst), dtype=np.complex128)
    for d, hm, b in zip(doms, hams, locs):
        out = torch.zeros((d.np_local, ld), dtype=tdt, device=cuda)
        hm.ham.apply(b, out, nst=nst, terms=lib.TERM_KINETIC | lib.TERM_LOCAL_POTENTIAL, set_bc=False)
        hm.ham.projector_ket(total, out, nst=nst)
        got = out.cpu().numpy()[:, :nst]
        assert np.max(np.abs(got - ref[d.inner_rows])) <= tol * np.max(np.abs(ref))
        full[d.inner_rows] = got
    assert rel_maxnorm_per_state(full, _oracle(m, w, v, proj).apply(psi)) <= (1e-12 if dtype == "c128" else 2e-5)


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_partitioned_hpsi_with_projector_phases_equals_global(cuda, dtype):
    """k != 0 on partitions: DomainHamiltonian restricts the global projector
    phases to each partition's sphere points; the summed projection shares
    and each partition's ket give the global H psi with phases."""
    import torch
    from hpsi import lib
    from hpsi.domain import DomainHamiltonian, partition_z
    from hpsi.stencil import laplacian_weights, star_points
    nst, ld, nparts = 16, 16, 3
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    m, v, proj, psi = small_sphere_system(seed=43, nst=nst, radius=4.5, natoms=4)
    rng = np.random.default_rng(44)
    ph = [np.exp(1j * rng.uniform(0, 2 * np.pi, len(mp))) for mp in proj.maps]
    w = laplacian_weights(m.spacing)
    H = lib.Hamiltonian(lib.DeviceMesh(m), w, star_points(), v=v, projectors=proj)
    H.set_projector_phases(ph)
    x = torch.from_numpy(np.ascontiguousarray(psi)).to(cuda).to(tdt)
    y = torch.zeros((m.np, ld), dtype=tdt, device=cuda)
    H.apply(x, y)
    ref = y.cpu().numpy()
    doms = partition_z(m, nparts)
    hams = [DomainHamiltonian(d, w, star_points(), v_global=v, projectors=proj, projector_phases=ph)
            for d in doms]
    locs = []
    for d in doms:
        b = d.local_batch(psi)
        b[d.np_local: d.np_local + d.np_ghost] = 0.0
        locs.append(torch.from_numpy(b).to(cuda).to(tdt))
    _exchange_on_one_gpu(doms, locs, nst)
    shares = []
    for hm, b in zip(hams, locs):
        pr = torch.zeros((hm.nprojections, ld), dtype=tdt, device=cuda)
        hm.ham.projector_bra(b, pr)
        shares.append(pr)
    total = torch.stack(shares).sum(0)
    tol = 1e-13 if dtype == "c128" else 2e-6
    for d, hm, b in zip(doms, hams, locs):
        out = torch.zeros((d.np_local, ld), dtype=tdt, device=cuda)
        hm.ham.apply(b, out, terms=lib.TERM_KINETIC | lib.TERM_LOCAL_POTENTIAL, set_bc=False)
        hm.ham.projector_ket(total, out)
        got = out.cpu().numpy()
        assert np.max(np.abs(got - ref[d.inner_rows])) <= tol * np.max(np.abs(ref))


def test_projector_bra_rejects_host_buffers(cuda):
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    m, v, proj, psi = small_sphere_system(seed=31, nst=4)
    H = lib.Hamiltonian(lib.DeviceMesh(m), laplacian_weights(m.spacing), star_points(), v=v, projectors=proj)
    x = torch.zeros((m.np_part, 4), dtype=torch.complex128, device=cuda)
    with pytest.raises(lib.HpsiError):
        H.projector_bra(x, torch.zeros((H.nprojections(), 4), dtype=torch.complex128))


@pytest.mark.parametrize("nparts,ld,dtype", [(2, 16, "c128"), (3, 16, "c128"), (3, 32, "c64")])
def test_partitioned_taylor_step_equals_global(cuda, nparts, ld, dtype):
    """Order-4 Taylor step on partitions, level by level in Horner form
    (hpsi_apply_h_horner without the KB term, the projection shares of every
    partition summed on the device, hpsi_projector_ket with a = -i dt / k),
    each level after a ghost exchange: equals the global hpsi_taylor_step."""
    import torch
    from hpsi import lib
    from hpsi.domain import DomainHamiltonian, partition_z
    from hpsi.stencil import laplacian_weights, star_points
    nst, dt, order = 16, 0.02, 4
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    m, v, proj, psi = small_sphere_system(seed=37, nst=nst, radius=4.5, natoms=4)
    g = np.zeros((m.np_part, ld), dtype=np.complex128)
    g[:, :nst] = psi
    w = laplacian_weights(m.spacing)
    H = lib.Hamiltonian(lib.DeviceMesh(m), w, star_points(), v=v, projectors=proj)
    xg = torch.from_numpy(g).to(cuda).to(tdt)
    H.taylor_step(xg, dt, order=order, nst=nst)
    ref = xg.cpu().numpy()[: m.np, :nst]
    doms = partition_z(m, nparts)
    hams = [DomainHamiltonian(d, w, star_points(), v_global=v, projectors=proj) for d in doms]
    psis = []
    for d in doms:
        b = d.local_batch(g)
        b[d.np_local: d.np_local + d.np_ghost] = 0.0
        psis.append(torch.from_numpy(b).to(cuda).to(tdt))
    work = [[torch.zeros_like(p), torch.zeros_like(p)] for p in psis]
    terms = lib.TERM_KINETIC | lib.TERM_LOCAL_POTENTIAL
    xs = list(psis)
    for k in range(order, 0, -1):
        a = -1j * dt / k
        _exchange_on_one_gpu(doms, xs, nst)
        shares = []
        for hm, x in zip(hams, xs):
            pr = torch.zeros((hm.nprojections, ld), dtype=tdt, device=cuda)
            hm.ham.projector_bra(x, pr)
            shares.append(pr)
        total = torch.stack(shares).sum(0)
        outs = []
        for p, (hm, x) in enumerate(zip(hams, xs)):
            out = work[p][(order - k) % 2] if k > 1 else psis[p]
            hm.ham.apply_horner(x, psis[p], out, a, nst=nst, terms=terms, set_bc=False)
            hm.ham.projector_ket(total, out, nst=nst, a=a)
            outs.append(out)
        xs = outs
    tol = 1e-12 if dtype == "c128" else 1e-5
    full = np.zeros((m.np, nst), dtype=np.complex128)
    for d, p in zip(doms, psis):
        got = p.cpu().numpy()[: d.np_local, :nst]
        assert np.max(np.abs(got - ref[d.inner_rows])) <= tol * np.max(np.abs(ref))
        full[d.inner_rows] = got
    oref = _oracle(m, w, v, proj).taylor(psi, dt, order=order)
    assert rel_maxnorm_per_state(full, oref) <= (1e-12 if dtype == "c128" else 2e-5)


def test_apply_h_horner_matches_apply(cuda):
    """hpsi_apply_h_horner: out = psi0 + a H psi (every term), and it refuses
    out aliasing psi."""
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    m, v, proj, psi = small_sphere_system(seed=41, nst=8, radius=4.0, natoms=3)
    H = lib.Hamiltonian(lib.DeviceMesh(m), laplacian_weights(m.spacing), star_points(), v=v, projectors=proj)
    x = torch.from_numpy(psi).to(cuda)
    p0 = torch.from_numpy(np.roll(psi, 1, axis=1)).to(cuda)
    hx = torch.zeros((m.np, 8), dtype=torch.complex128, device=cuda)
    H.apply(x, hx)
    a = 0.3 - 0.7j
    out = torch.zeros((m.np, 8), dtype=torch.complex128, device=cuda)
    H.apply_horner(x, p0, out, a)
    want = p0[: m.np] + a * hx
    assert (out - want).abs().max().item() <= 1e-13 * want.abs().max().item()
    with pytest.raises(lib.HpsiError):
        H.apply_horner(x, p0, x, a)


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_domain_hamiltonian_methods_single_partition(cuda, dtype):
    """DomainHamiltonian.apply and .taylor_step (the classes' own paths:
    apply_partitioned, taylor_partitioned, the projection buffer) on one
    partition, where no exchange or all-reduce runs: equal the global
    hpsi_apply_h and hpsi_taylor_step."""
    import torch
    from hpsi import lib
    from hpsi.domain import DomainHamiltonian, partition_z
    from hpsi.stencil import laplacian_weights, star_points
    nst, ld, dt = 16, 16, 0.02
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    m, v, proj, psi = small_sphere_system(seed=53, nst=nst, radius=4.5, natoms=4)
    w = laplacian_weights(m.spacing)
    H = lib.Hamiltonian(lib.DeviceMesh(m), w, star_points(), v=v, projectors=proj)
    x = torch.from_numpy(psi).to(cuda).to(tdt)
    y = torch.zeros((m.np, ld), dtype=tdt, device=cuda)
    H.apply(x, y)
    d = partition_z(m, 1)[0]
    hm = DomainHamiltonian(d, w, star_points(), v_global=v, projectors=proj)
    xl = torch.from_numpy(d.local_batch(psi)).to(cuda).to(tdt)
    yl = torch.zeros((d.np_local, ld), dtype=tdt, device=cuda)
    hm.apply(xl, yl)
    tol = 1e-13 if dtype == "c128" else 2e-6
    ref = y.cpu().numpy()
    assert np.max(np.abs(yl.cpu().numpy() - ref[d.inner_rows])) <= tol * np.max(np.abs(ref))
    H.taylor_step(x, dt)
    hm.taylor_step(xl, dt)
    ref_t = x.cpu().numpy()[: m.np]
    tol_t = 1e-12 if dtype == "c128" else 1e-5
    got_t = xl.cpu().numpy()[: d.np_local]
    assert np.max(np.abs(got_t - ref_t[d.inner_rows])) <= tol_t * np.max(np.abs(ref_t))


@pytest.mark.parametrize("dtype,horner", [("c128", False), ("c128", True), ("c64", False)])
def test_inner_outer_split_reads_no_ghost_and_covers_every_row(cuda, dtype, horner):
    """hpsi_apply_h_points / hpsi_apply_h_horner_points on the partitions of a
    slab decomposition: the INNER part runs on batches whose ghost rows are
    NaN (the exchange still in flight) and must not read them; the ghost rows
    are then filled and the OUTER part runs; together they equal the ALL pass
    on the filled batch bit for bit (the same arithmetic per output row) and
    the global H psi."""
    import torch
    from hpsi import lib
    from hpsi.domain import POINTS_INNER, POINTS_OUTER, DomainHamiltonian, partition_z
    from hpsi.stencil import laplacian_weights, star_points
    nst = 16
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    m, v, proj, psi = small_sphere_system(seed=59, nst=nst, radius=5.0, natoms=0)
    w = laplacian_weights(m.spacing)
    terms = lib.TERM_KINETIC | lib.TERM_LOCAL_POTENTIAL
    H = lib.Hamiltonian(lib.DeviceMesh(m), w, star_points(), v=v)
    xg = torch.from_numpy(np.ascontiguousarray(psi)).to(cuda).to(tdt)
    yg = torch.zeros((m.np, nst), dtype=tdt, device=cuda)
    H.apply(xg, yg, terms=terms)
    ref = yg.cpu().numpy()
    doms = partition_z(m, 3)
    hams = [DomainHamiltonian(d, w, star_points(), v_global=v) for d in doms]
    locs = [torch.from_numpy(d.local_batch(psi)).to(cuda).to(tdt) for d in doms]
    for d, b in zip(doms, locs):
        b[d.np_local: d.np_local + d.np_ghost] = float("nan")
    a = 0.3 - 0.2j
    outs = []
    for d, hm, b in zip(doms, hams, locs):
        y = torch.zeros((d.np_local, nst), dtype=tdt, device=cuda)
        if horner:
            p0 = b[: d.np_local].clone()
            hm.ham.apply_horner(b, p0, y, a, terms=terms, set_bc=False, points=POINTS_INNER)
        else:
            hm.ham.apply(b, y, terms=terms, set_bc=False, points=POINTS_INNER)
        outs.append(y)
    _exchange_on_one_gpu(doms, locs, nst)
    tol = 1e-13 if dtype == "c128" else 2e-6
    n_inner = 0
    for d, hm, b, y in zip(doms, hams, locs, outs):
        ninner_rows = int(torch.count_nonzero(y.abs().sum(1)).item())
        n_inner += ninner_rows
        if horner:
            p0 = b[: d.np_local].clone()
            hm.ham.apply_horner(b, p0, y, a, terms=terms, set_bc=False, points=POINTS_OUTER)
            full = torch.zeros_like(y)
            hm.ham.apply_horner(b, p0, full, a, terms=terms, set_bc=False)
        else:
            hm.ham.apply(b, y, terms=terms, set_bc=False, points=POINTS_OUTER)
            full = torch.zeros_like(y)
            hm.ham.apply(b, full, terms=terms, set_bc=False)
        assert not torch.isnan(y).any()
        assert torch.equal(y, full)
        if not horner:
            assert np.max(np.abs(y.cpu().numpy() - ref[d.inner_rows])) <= tol * np.max(np.abs(ref))
    # the inner part holds a real share of the points (the overlap has work to hide the exchange)
    assert n_inner >= m.np // 10


def test_points_reject_kb_term(cuda):
    import torch
    from hpsi import lib
    from hpsi.domain import POINTS_INNER
    from hpsi.stencil import laplacian_weights, star_points
    m, v, proj, psi = small_sphere_system(seed=61, nst=4)
    H = lib.Hamiltonian(lib.DeviceMesh(m), laplacian_weights(m.spacing), star_points(), v=v, projectors=proj)
    x = torch.from_numpy(psi).to(cuda)
    y = torch.zeros((m.np, 4), dtype=torch.complex128, device=cuda)
    with pytest.raises(lib.HpsiError):
        H.apply(x, y, points=POINTS_INNER)
