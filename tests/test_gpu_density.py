"""Density accumulation (density_calc_accumulate) on the GPU against the oracle,
alone and after a Taylor step (the density of the propagated states)."""
import numpy as np
import pytest

from helpers import small_sphere_system

pytestmark = pytest.mark.gpu


def _setup(mesh, v=None, proj=None):
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    dm = lib.DeviceMesh(mesh)
    ham = lib.Hamiltonian(dm, laplacian_weights(mesh.spacing), star_points(), v=v, projectors=proj)
    return dm, ham


@pytest.mark.parametrize("dtype,ld,nst", [(np.complex128, 8, 8), (np.complex128, 16, 11), (np.complex64, 16, 16)])
def test_density_matches_oracle(cuda, dtype, ld, nst):
    import torch
    from oracle import oracle as O
    m, v, proj, psi = small_sphere_system(seed=71, nst=nst)
    dm, ham = _setup(m, v, proj)
    rng = np.random.default_rng(72)
    w = rng.uniform(0.0, 2.0, nst)
    host = np.zeros((m.np_part, ld), dtype=dtype)
    host[:, :nst] = psi
    x = torch.from_numpy(host).to(cuda)
    rho = dm.density(x, w, nst=nst)
    ref = O.density_accumulate(m, host[:, :nst].astype(np.complex128), w)
    got = rho.cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))
    # accumulate into the existing density
    rho2 = dm.density(x, w, rho=rho, accumulate=True, nst=nst)
    assert np.max(np.abs(rho2.cpu().numpy() - 2 * ref)) <= 1e-13 * np.max(np.abs(ref))


def test_density_of_propagated_states(cuda):
    """propagation_ops_elec_fuse_density_exp_apply: exp(-i dt H) then density."""
    import torch
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O
    m, v, proj, psi = small_sphere_system(seed=73, nst=8)
    dm, ham = _setup(m, v, proj)
    w = np.full(8, 2.0)
    x = torch.from_numpy(psi).to(cuda)
    ham.taylor_step(x, 0.02)
    rho = dm.density(x, w)
    P = O.Projectors(proj.maps, proj.mats, proj.scals)
    ref_psi = O.Hamiltonian(m, laplacian_weights(m.spacing), star_points(), v=v, projectors=P).taylor(psi, 0.02)
    ref = O.density_accumulate(m, ref_psi, w)
    assert np.max(np.abs(rho.cpu().numpy() - ref)) <= 1e-12 * np.max(np.abs(ref))
    # the density integrates to sum_i w_i ||psi_i||^2 of the propagated states (the
    # Taylor series is not unitary: the norms move at the 1e-3 level here)
    norms = m.vol_pp * np.sum(np.abs(ref_psi[: m.np]) ** 2, axis=0)
    assert abs(m.vol_pp * float(rho.sum()) - float(w @ norms)) <= 1e-12 * float(w @ norms)


@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("dtype,nst,ld", [("c128", 16, 16), ("c64", 32, 32), ("c128", 6, 6), ("c64", 40, 48)])
def test_taylor_step_density(cuda, dtype, nst, ld, fused, monkeypatch):
    """hpsi_taylor_step_density: the propagated batch equals hpsi_taylor_step's
    bit for bit, and the density equals the density kernel on the propagated
    batch and the oracle's step + density.  Both forms: the density pass after
    the step (default), and the density fused into the last Horner pass with
    the KB-covered rows from the ket's final values (widths the blocked pass
    does not take use the density pass in either form)."""
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O
    monkeypatch.setenv("HPSI_FUSED_DENSITY", "1" if fused else "0")
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    m, v, proj, psi = small_sphere_system(seed=53, nst=nst, radius=4.0, natoms=3)
    w = laplacian_weights(m.spacing)
    dm = lib.DeviceMesh(m)
    H = lib.Hamiltonian(dm, w, star_points(), v=v, projectors=proj)
    g = np.zeros((m.np_part, ld), dtype=np.complex128)
    g[:, :nst] = psi
    wt = np.random.default_rng(54).uniform(0.5, 2.0, nst)
    a = torch.from_numpy(g).to(cuda).to(tdt)
    b = a.clone()
    dt = 0.01
    H.taylor_step(a, dt, nst=nst)
    rho = H.taylor_step_density(b, dt, wt, nst=nst)
    assert torch.equal(a[: m.np], b[: m.np])
    ref = dm.density(a, wt, nst=nst)
    tol = 1e-13
    assert torch.max(torch.abs(rho - ref)).item() <= tol * torch.max(ref).item()
    rho2 = H.taylor_step_density(b.clone(), dt, wt, rho=rho.clone(), accumulate=True, nst=nst)
    ref2 = dm.density(a, wt, nst=nst)
    H.taylor_step(a, dt, nst=nst)
    ref2 = dm.density(a, wt, rho=ref2, accumulate=True, nst=nst)
    assert torch.max(torch.abs(rho2 - ref2)).item() <= tol * torch.max(ref2).item()
    if dtype == "c128":
        P = O.Projectors(proj.maps, proj.mats, proj.scals)
        y = O.Hamiltonian(m, w, star_points(), v=v, projectors=P).taylor(psi, dt)
        yp = np.zeros((m.np_part, nst), dtype=np.complex128)
        yp[: m.np] = y
        ro = O.density_accumulate(m, yp, wt)
        assert np.max(np.abs(rho.cpu().numpy() - ro)) <= 1e-12 * np.max(ro)
