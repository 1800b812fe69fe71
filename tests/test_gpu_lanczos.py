"""Lanczos exponential (exponential_lanczos_batch) against the oracle's restatement."""
import numpy as np
import pytest

from helpers import rel_maxnorm_per_state, small_sphere_system

pytestmark = pytest.mark.gpu


def _setup(seed, nst):
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O
    m, v, proj, psi = small_sphere_system(seed=seed, nst=nst)
    w = laplacian_weights(m.spacing)
    dm = lib.DeviceMesh(m)
    ham = lib.Hamiltonian(dm, w, star_points(), v=v, projectors=proj)
    P = O.Projectors(proj.maps, proj.mats, proj.scals)
    H = O.Hamiltonian(m, w, star_points(), v=v, projectors=P)
    return m, psi, ham, H


@pytest.mark.parametrize("dt,tol", [(0.02, 1e-10), (0.1, 1e-8)])
def test_lanczos_matches_oracle(cuda, dt, tol):
    import torch
    from oracle import oracle as O
    m, psi, ham, H = _setup(81, 6)
    ref, mref, rref = O.lanczos(H, psi, dt, max_order=40, tol=tol)
    x = torch.from_numpy(psi.copy()).to(cuda)
    mgpu, rgpu = ham.lanczos_step(x, dt, max_order=40, tol=tol)
    assert mgpu == mref
    assert rgpu < tol
    assert rel_maxnorm_per_state(x.cpu().numpy()[: m.np], ref) <= 1e-11


def test_lanczos_agrees_with_taylor_for_small_dt(cuda):
    import torch
    m, psi, ham, H = _setup(83, 4)
    x = torch.from_numpy(psi.copy()).to(cuda)
    y = x.clone()
    ham.lanczos_step(x, 0.005, max_order=30, tol=1e-12)
    ham.taylor_step(y, 0.005, order=4)  # Taylor error O((dt E)^5 / 120)
    assert rel_maxnorm_per_state(x.cpu().numpy()[: m.np], y.cpu().numpy()[: m.np]) <= 2e-4


def test_lanczos_stable_beyond_taylor_limit(cuda):
    """dt far past the Taylor-4 stability bound: the Lanczos step keeps the norms."""
    import torch
    m, psi, ham, H = _setup(85, 4)
    x = torch.from_numpy(psi.copy()).to(cuda)
    n0 = np.sum(np.abs(psi[: m.np]) ** 2, axis=0)
    it, res = ham.lanczos_step(x, 0.5, max_order=64, tol=1e-6)
    n1 = np.sum(np.abs(x.cpu().numpy()[: m.np]) ** 2, axis=0)
    assert res < 1e-6
    assert np.max(np.abs(n1 - n0) / n0) <= 1e-6


def test_lanczos_null_states_and_fp32_rejected(cuda):
    """All-zero states: nothing to expand (the reference returns early too);
    complex64 batches are refused (the Lanczos step is FP64 only)."""
    import torch
    from hpsi import lib
    m, psi, ham, H = _setup(87, 4)
    z = torch.zeros((m.np_part, 4), dtype=torch.complex128, device=cuda)
    assert ham.lanczos_step(z, 0.05) == (0, 0.0)
    assert not z.abs().max().item()
    x32 = torch.from_numpy(psi.copy()).to(cuda).to(torch.complex64)
    with pytest.raises(lib.HpsiError):
        ham.lanczos_step(x32, 0.05)
