"""The FP64 stencil pass with its in-plane arms on the FP64 tensor cores
(banded DMMA products, csrc/stencil_mma.cu), selected by the shape override.

Against the oracle at the FP64 parity tolerance: H psi on a KB sphere (one
and five state chunks), the raw map (set_bc = False), a box with several z
blocks per column, Bloch-phase periodic images, a Taylor step (Horner passes)
and the FP64 observables of its first pass; against the default pass with a
laser field on (the field term rides on the local potential)."""
import numpy as np
import pytest

from helpers import rel_maxnorm_per_state, small_sphere_system

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
VAR = "HPSI_PASS_SHAPE64"
MMA = "8,2,{zb},9,1,2,0,8,0,0,1"


def _ham(m, v=None, proj=None):
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    w = laplacian_weights(m.spacing)
    dm = lib.DeviceMesh(m)
    return dm, lib.Hamiltonian(dm, w, star_points(), v=v, projectors=proj), w


def _oracle(m, w, v=None, proj=None, **kw):
    from hpsi.stencil import star_points
    from oracle import oracle as O
    P = O.Projectors(proj.maps, proj.mats, proj.scals) if proj is not None else None
    return O.Hamiltonian(m, w, star_points(), v=v, projectors=P, **kw)


@pytest.mark.parametrize("nst", [8, 40])
def test_mma_pass_sphere_apply_taylor(cuda, monkeypatch, nst):
    import torch
    m, v, proj, psi = small_sphere_system(seed=91, nst=nst, radius=4.5, natoms=3)
    dm, H, w = _ham(m, v, proj)
    O = _oracle(m, w, v, proj)
    x = torch.from_numpy(psi).to(cuda)
    monkeypatch.setenv(VAR, MMA.format(zb=0))
    y = torch.zeros((m.np, nst), dtype=torch.complex128, device=cuda)
    H.apply(x, y)
    assert rel_maxnorm_per_state(y.cpu().numpy(), O.apply(psi)) <= TOL64
    yr = torch.zeros_like(y)
    H.apply(x, yr, set_bc=False)
    assert rel_maxnorm_per_state(yr.cpu().numpy(), O.apply(psi)) <= TOL64  # boundary rows of psi are zero
    xt = x.clone()
    H.taylor_step(xt, 0.01)
    assert rel_maxnorm_per_state(xt[: m.np].cpu().numpy(), O.taylor(psi, 0.01)) <= TOL64
    xo = x.clone()
    e, d, n = H.taylor_step(xo, 0.01, observables=True)
    assert torch.equal(xo, xt)  # the observables do not change the step
    assert H.status() == 0
    # observables of the first pass against the default pass
    monkeypatch.delenv(VAR)
    xd = x.clone()
    e0, d0, n0 = H.taylor_step(xd, 0.01, observables=True)
    for a, b in ((e, e0), (d, d0), (n, n0)):
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
    assert rel_maxnorm_per_state(xd.cpu().numpy(), xt.cpu().numpy()) <= TOL64


@pytest.mark.parametrize("zb", [0, 8, 16])
def test_mma_pass_box_zblocks(cuda, monkeypatch, zb):
    import torch
    from hpsi import fixtures
    from hpsi.mesh import index_box_mesh
    rng = np.random.default_rng(92)
    m = index_box_mesh((36, 20, 40), 0.25)
    v = fixtures.soft_coulomb(m, rng)
    psi = fixtures.random_states(m, 16, rng, orthonormal=False)
    dm, H, w = _ham(m, v)
    monkeypatch.setenv(VAR, MMA.format(zb=zb))
    x = torch.from_numpy(psi).to(cuda)
    y = torch.zeros((m.np, 16), dtype=torch.complex128, device=cuda)
    H.apply(x, y)
    assert rel_maxnorm_per_state(y.cpu().numpy(), _oracle(m, w, v).apply(psi)) <= TOL64


def test_mma_pass_bloch_phase(cuda, monkeypatch):
    import torch
    from hpsi import fixtures
    from hpsi.mesh import index_box_mesh
    rng = np.random.default_rng(93)
    m = index_box_mesh((12, 10, 8), 0.3, periodic=True)
    v = fixtures.soft_coulomb(m, rng)
    psi = fixtures.random_states(m, 8, rng, orthonormal=False)
    k = np.array([0.3, -0.2, 0.5])
    pc = np.exp(1j * ((m.x[m.np:] - m.x[m.per_inner]) @ k))
    dm, H, w = _ham(m, v)
    H.set_phase_corr(pc)
    monkeypatch.setenv(VAR, MMA.format(zb=0))
    x = torch.from_numpy(psi).to(cuda)
    y = torch.zeros((m.np, 8), dtype=torch.complex128, device=cuda)
    H.apply(x, y)
    ref = _oracle(m, w, v, bc="periodic", phase_corr=pc).apply(psi)
    assert rel_maxnorm_per_state(y.cpu().numpy(), ref) <= TOL64


def test_mma_pass_laser_field(cuda, monkeypatch):
    import torch
    m, v, proj, psi = small_sphere_system(seed=94, nst=16, radius=4.0, natoms=2)
    dm, H, w = _ham(m, v, proj)
    H.set_field((0.3, -0.5, 0.8), 0.05)
    x = torch.from_numpy(psi).to(cuda)
    monkeypatch.delenv(VAR, raising=False)
    y0 = torch.zeros((m.np, 16), dtype=torch.complex128, device=cuda)
    H.apply(x, y0)
    monkeypatch.setenv(VAR, MMA.format(zb=0))
    y1 = torch.zeros_like(y0)
    H.apply(x, y1)
    assert rel_maxnorm_per_state(y1.cpu().numpy(), y0.cpu().numpy()) <= TOL64


def test_mma_pass_fp32_rejected(cuda, monkeypatch):
    """The tensor-core pass is FP64 only: the FP32 override is refused."""
    import torch
    from hpsi import lib
    m, v, proj, psi = small_sphere_system(seed=95, nst=16)
    dm, H, w = _ham(m, v, proj)
    monkeypatch.setenv("HPSI_PASS_SHAPE32", "16,2,0,9,1,2,1,8,0,0,1")
    x = torch.from_numpy(psi.astype(np.complex64)).to(cuda)
    y = torch.zeros((m.np, 16), dtype=torch.complex64, device=cuda)
    with pytest.raises(lib.HpsiError):
        H.apply(x, y)
