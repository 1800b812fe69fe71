"""Grouped systems (one persistent launch per pass) and the autotuner."""
import numpy as np
import pytest

from helpers import rel_maxnorm_per_state

pytestmark = pytest.mark.gpu


def _system(seed, n, nst, natoms):
    from hpsi import fixtures
    from hpsi.mesh import index_box_mesh
    rng = np.random.default_rng(seed)
    m = index_box_mesh((n, n + 1, n - 1), 0.25)
    v = fixtures.soft_coulomb(m, rng)
    proj = fixtures.kb_projectors(m, natoms, rng, radius=0.8, min_dist=0.6, place_radius=0.8) if natoms else None
    psi = fixtures.random_states(m, nst, rng)
    return m, v, proj, psi


def test_group_matches_single_systems(cuda):
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    specs = [(1, 12, 4, 2), (2, 17, 7, 0), (3, 9, 16, 3), (4, 21, 5, 1), (5, 14, 12, 2)]
    hams, xs, refs = [], [], []
    for seed, n, nst, natoms in specs:
        m, v, proj, psi = _system(seed, n, nst, natoms)
        dm = lib.DeviceMesh(m)
        ham = lib.Hamiltonian(dm, laplacian_weights(m.spacing), star_points(), v=v, projectors=proj)
        ld = 1 << (nst - 1).bit_length()
        x = torch.zeros((m.np_part, ld), dtype=torch.complex128, device=cuda)
        x[:, :nst] = torch.from_numpy(psi)
        r = x.clone()
        for _ in range(3):
            ham.taylor_step(r, 0.02, nst=nst)
        hams.append((dm, ham))
        xs.append(x)
        refs.append(r)
    g = lib.Group([h for _, h in hams])
    for graph in (False, True):
        ys = [x.clone() for x in xs]
        g.taylor_steps(ys, 3, 0.02, graph=graph)
        torch.cuda.synchronize()
        for y, r, (seed, n, nst, natoms) in zip(ys, refs, specs):
            np_ = r.shape[0]
            assert rel_maxnorm_per_state(y.cpu().numpy()[:, :nst], r.cpu().numpy()[:, :nst]) <= 1e-14
    g.close()


def test_autotune_keeps_results(cuda):
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    m, v, proj, psi = _system(7, 20, 8, 2)
    dm = lib.DeviceMesh(m)
    ham = lib.Hamiltonian(dm, laplacian_weights(m.spacing), star_points(), v=v, projectors=proj)
    x = torch.from_numpy(psi).to(cuda)
    y0 = torch.zeros((m.np, 8), dtype=torch.complex128, device=cuda)
    ham.apply(x, y0)
    shape, ms = ham.autotune(lib.HPSI_C128, 8)
    assert shape["sc"] in (1, 2, 4, 8) and ms > 0
    y1 = torch.zeros_like(y0)
    ham.apply(x, y1)
    assert rel_maxnorm_per_state(y1.cpu().numpy(), y0.cpu().numpy()) <= 1e-14
    x32 = x.to(torch.complex64)
    shape32, _ = ham.autotune(lib.HPSI_C64, 8)
    assert shape32["sc"] in (2, 4, 8)


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_group_blocked_pass_matches_single_systems(cuda, dtype):
    """Every width a multiple of the blocked pass's chunk (8 complex128 / 16
    complex64 states): the grouped launch runs the blocked pass kernel."""
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    chunk = 8 if dtype == "c128" else 16
    specs = [(11, 13, 5, 2), (12, 18, chunk + 3, 0), (13, 10, 2 * chunk, 3), (14, 22, 3, 1)]
    hams, xs, refs, nsts = [], [], [], []
    for seed, n, nst, natoms in specs:
        m, v, proj, psi = _system(seed, n, nst, natoms)
        dm = lib.DeviceMesh(m)
        ham = lib.Hamiltonian(dm, laplacian_weights(m.spacing), star_points(), v=v, projectors=proj)
        ld = chunk * ((nst + chunk - 1) // chunk)
        x = torch.zeros((m.np_part, ld), dtype=tdt, device=cuda)
        x[:, :nst] = torch.from_numpy(psi).to(tdt)
        r = x.clone()
        for _ in range(3):
            ham.taylor_step(r, 0.02)
        hams.append((dm, ham))
        xs.append(x)
        refs.append(r)
        nsts.append(nst)
    g = lib.Group([h for _, h in hams])
    tol = 1e-13 if dtype == "c128" else 1e-6
    for graph in (False, True):
        ys = [x.clone() for x in xs]
        g.taylor_steps(ys, 3, 0.02, graph=graph)
        torch.cuda.synchronize()
        for y, r, nst in zip(ys, refs, nsts):
            a = y.cpu().numpy()[:, :nst].astype(np.complex128)
            b = r.cpu().numpy()[:, :nst].astype(np.complex128)
            assert rel_maxnorm_per_state(a, b) <= tol
    g.close()


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_group_with_laser_field_matches_single_systems(cuda, dtype):
    """Systems with a laser field in the group (the persistent pass with the
    field term; without a field in any system it takes the field-free form):
    each system as its own Taylor steps with the same field."""
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    chunk = 8 if dtype == "c128" else 16
    specs = [(21, 14, chunk, 2), (22, 17, 2 * chunk, 0), (23, 11, chunk, 1)]
    fields = [((0.3, -0.5, 0.8), 0.05), None, ((0.0, 0.0, 1.0), -0.02)]
    hams, xs, refs = [], [], []
    for (seed, n, nst, natoms), fld in zip(specs, fields):
        m, v, proj, psi = _system(seed, n, nst, natoms)
        dm = lib.DeviceMesh(m)
        ham = lib.Hamiltonian(dm, laplacian_weights(m.spacing), star_points(), v=v, projectors=proj)
        if fld is not None:
            ham.set_field(*fld)
        x = torch.zeros((m.np_part, nst), dtype=tdt, device=cuda)
        x[:, :nst] = torch.from_numpy(psi).to(tdt)
        r = x.clone()
        for _ in range(3):
            ham.taylor_step(r, 0.02)
        hams.append((dm, ham))
        xs.append(x)
        refs.append(r)
    g = lib.Group([h for _, h in hams])
    tol = 1e-13 if dtype == "c128" else 1e-6
    ys = [x.clone() for x in xs]
    g.taylor_steps(ys, 3, 0.02)
    torch.cuda.synchronize()
    for y, r in zip(ys, refs):
        a = y.cpu().numpy().astype(np.complex128)
        b = r.cpu().numpy().astype(np.complex128)
        assert rel_maxnorm_per_state(a, b) <= tol
    g.close()
