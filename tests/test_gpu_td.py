"""Time propagation (exponential midpoint + laser) against the FP64 oracle."""
import numpy as np
import pytest

from helpers import rel_maxnorm_per_state, small_sphere_system

pytestmark = pytest.mark.gpu

LASER = dict(E0=0.05, omega=0.057, T=0.8)


def _systems(seed=37, nst=4):
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O
    m, v, proj, psi = small_sphere_system(seed=seed, nst=nst)
    w = laplacian_weights(m.spacing)
    dm = lib.DeviceMesh(m)
    ham = lib.Hamiltonian(dm, w, star_points(), v=v, projectors=proj)
    P = O.Projectors(proj.maps, proj.mats, proj.scals)
    H = O.Hamiltonian(m, w, star_points(), v=v.copy(), projectors=P)
    return m, v, psi, dm, ham, H


@pytest.mark.parametrize("graph", [False, True])
def test_td_fp64_matches_oracle(cuda, graph):
    import torch
    from oracle import oracle as O
    m, v, psi, dm, ham, H = _systems()
    nsteps, dt = 40, 0.02
    ref, Er, Dr, Nr = O.td_propagate(H, v, psi, nsteps, dt, **LASER)
    x = torch.from_numpy(psi.copy()).to(cuda)
    E, D, N = ham.td_propagate(x, nsteps, dt, graph=graph, **LASER)
    got = x.cpu().numpy()[: m.np]
    assert rel_maxnorm_per_state(got, ref) <= 1e-11
    assert np.max(np.abs(E - Er) / np.abs(Er)) <= 1e-11
    assert np.max(np.abs(N - Nr) / Nr) <= 1e-12
    assert np.max(np.abs(D - Dr)) <= 1e-11 * np.max(np.abs(Nr))
    assert np.ptp(D) > 1e-6  # the laser moves the dipole


def test_td_fp32_observables_close_to_fp64(cuda):
    import torch
    m, v, psi, dm, ham, H = _systems(seed=43, nst=8)
    nsteps, dt = 100, 0.02
    x64 = torch.from_numpy(psi.copy()).to(cuda)
    x32 = torch.from_numpy(psi.astype(np.complex64)).to(cuda)
    E64, D64, N64 = ham.td_propagate(x64, nsteps, dt, **LASER)
    E32, D32, N32 = ham.td_propagate(x32, nsteps, dt, **LASER)
    assert np.max(np.abs(E32 - E64) / np.abs(E64)) <= 1e-5
    assert np.max(np.abs(D32 - D64)) <= 1e-5 * np.max(np.abs(N64))


def test_td_runaway_detected(cuda):
    import torch
    from hpsi import lib
    m, v, psi, dm, ham, H = _systems(nst=2)
    x = torch.from_numpy(psi.copy()).to(cuda)
    with pytest.raises(lib.HpsiError) as e:
        ham.td_propagate(x, 5, 1.0, graph=False)  # dt far beyond the Taylor stability limit
    assert e.value.status == 8


@pytest.mark.parametrize("graph", [False, True])
def test_td_etrs_matches_oracle(cuda, graph):
    """ETRS steps (two half-step exponentials with the fields of t_n and t_n+1)."""
    import torch
    from oracle import oracle as O
    m, v, psi, dm, ham, H = _systems(seed=47)
    nsteps, dt = 30, 0.02
    ref, Er, Dr, Nr = O.td_propagate(H, v, psi, nsteps, dt, propagator="etrs", **LASER)
    x = torch.from_numpy(psi.copy()).to(cuda)
    E, D, N = ham.td_propagate(x, nsteps, dt, graph=graph, propagator="etrs", **LASER)
    got = x.cpu().numpy()[: m.np]
    assert rel_maxnorm_per_state(got, ref) <= 1e-11
    assert np.max(np.abs(E - Er) / np.abs(Er)) <= 1e-11
    assert np.max(np.abs(N - Nr) / Nr) <= 1e-12
    assert np.max(np.abs(D - Dr)) <= 1e-11 * np.max(np.abs(Nr))


def test_taylor_step_dual_outputs(cuda):
    """psib2 output of exponential_apply_batch: psi2 = exp(-i dt2 H) psi and
    psi = exp(-i dt H) psi from one call, against the oracle's Taylor step."""
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O
    from helpers import rel_maxnorm_per_state, small_sphere_system
    m, v, proj, psi = small_sphere_system(seed=29, nst=8)
    w = laplacian_weights(m.spacing)
    ham = lib.Hamiltonian(lib.DeviceMesh(m), w, star_points(), v=v, projectors=proj)
    H = O.Hamiltonian(m, w, star_points(), v=v, projectors=O.Projectors(proj.maps, proj.mats, proj.scals))
    x = torch.from_numpy(psi.copy()).to(cuda)
    x2 = torch.zeros((m.np, 16), dtype=torch.complex128, device=cuda)
    ham.taylor_step_dual(x, x2, 0.005, 0.01, order=4, nst=8)  # psi2 rows strided (ld 16)
    assert rel_maxnorm_per_state(x.cpu().numpy()[: m.np], H.taylor(psi, 0.005, 4)) <= 1e-12
    assert rel_maxnorm_per_state(x2.cpu().numpy()[:, :8], H.taylor(psi, 0.01, 4)) <= 1e-12
    with pytest.raises(lib.HpsiError):
        ham.taylor_step_dual(x, x, 0.005, 0.01)  # same storage
