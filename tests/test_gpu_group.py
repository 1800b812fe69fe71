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
