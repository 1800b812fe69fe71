"""GPU parity of both stencil-pass kernels against the FP64 CPU oracle.

The register-blocked pass (one real lane per thread, 16 x 8 tiles) serves
batches whose width is a multiple of its state chunk (8 complex states FP64,
16 FP32); its half-chunk form (64 bytes: 4 FP64, 8 FP32 states, two CTAs per
SM) serves widths that are a multiple of half a chunk only (FP64 12, FP32 24
below); the one-complex-per-thread pass serves the rest.  The kernels are
forced here through the shape override and compared with the oracle and with
each other: FP64 to 1e-12 relative max-norm per state, FP32 storage to 2e-5.
"""
import numpy as np
import pytest

from helpers import rel_maxnorm_per_state, small_sphere_system

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5

LEGACY = {"HPSI_PASS_SHAPE64": "4,2,0,0,0", "HPSI_PASS_SHAPE32": "8,4,0,0,0"}
# blocked pass: "chunk,ry,zb,group,1,rx,complex"
BLK_REAL = {"HPSI_PASS_SHAPE64": "8,2,{zb},3,1,2,0", "HPSI_PASS_SHAPE32": "16,4,{zb},1,1,2,0"}
BLK_CPLX = {"HPSI_PASS_SHAPE64": "8,2,{zb},9,1,2,1", "HPSI_PASS_SHAPE32": "16,2,{zb},3,1,2,1"}
# 64-byte chunks on 16 x 16 tiles, 1 x 4 cells
BLK_64B = {"HPSI_PASS_SHAPE64": "4,4,{zb},9,1,1,0", "HPSI_PASS_SHAPE32": "8,4,{zb},9,1,1,1"}
# 64-byte chunks on 16 x 8 tiles, 1 x 4 cells, 256 threads (two CTAs per SM)
BLK_2CTA = {"HPSI_PASS_SHAPE64": "4,4,{zb},9,1,1,0,8", "HPSI_PASS_SHAPE32": "8,4,{zb},9,1,1,1,8"}
PATHS = ["default", "blk_real", "blk_cplx", "blk_64b", "blk_2cta", "legacy"]


def _setup(mesh, v=None, proj=None):
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    w = laplacian_weights(mesh.spacing)
    pts = star_points()
    dm = lib.DeviceMesh(mesh)
    ham = lib.Hamiltonian(dm, w, pts, v=v, projectors=proj)
    return dm, ham, w, pts


def _oracle(mesh, w, pts, v=None, proj=None, bc="zero"):
    from oracle import oracle as O
    P = O.Projectors(proj.maps, proj.mats, proj.scals) if proj is not None else None
    return O.Hamiltonian(mesh, w, pts, v=v, projectors=P, bc=bc)


def _dev(x, cuda, ld, dtype):
    import torch
    out = np.zeros((x.shape[0], ld), dtype=dtype)
    out[:, : x.shape[1]] = x
    return torch.from_numpy(out).to(cuda)


def _set_path(monkeypatch, path, zb=0):
    if path == "default":
        for k in LEGACY:
            monkeypatch.delenv(k, raising=False)
        return
    env = {"legacy": LEGACY, "blk_real": BLK_REAL, "blk_cplx": BLK_CPLX, "blk_64b": BLK_64B,
           "blk_2cta": BLK_2CTA}[path]
    for k, v in env.items():
        monkeypatch.setenv(k, v.format(zb=zb))


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("dtype,ld,nst", [(np.complex128, 16, 13), (np.complex128, 8, 8),
                                          (np.complex64, 16, 11), (np.complex64, 32, 20),
                                          (np.complex128, 12, 10), (np.complex64, 24, 21)])
def test_apply_and_taylor(cuda, monkeypatch, path, dtype, ld, nst):
    import torch
    from hpsi import lib
    _set_path(monkeypatch, path)
    m, v, proj, psi = small_sphere_system(seed=41, nst=nst, radius=4.2, natoms=4)
    dm, ham, w, pts = _setup(m, v=v, proj=proj)
    o = _oracle(m, w, pts, v=v, proj=proj)
    tol = TOL64 if dtype == np.complex128 else TOL32
    x = _dev(psi, cuda, ld, dtype)
    y = torch.zeros((m.np, ld), dtype=x.dtype, device=cuda)
    ham.apply(x, y, nst=nst)
    got = y.cpu().numpy()[:, :nst].astype(np.complex128)
    assert rel_maxnorm_per_state(got, o.apply(psi)) <= tol
    e, d, n = ham.taylor_step(x, 0.02, order=4, nst=nst, observables=True)
    got = x.cpu().numpy()[: m.np, :nst].astype(np.complex128)
    assert rel_maxnorm_per_state(got, o.taylor(psi, 0.02, order=4)) <= tol
    h = o.apply(psi)
    dv = m.vol_pp
    e_ref = dv * np.real(np.sum(psi[: m.np].conj() * h, axis=0))
    n_ref = dv * np.sum(np.abs(psi[: m.np]) ** 2, axis=0)
    assert np.max(np.abs(e - e_ref) / np.abs(e_ref)) <= (1e-12 if dtype == np.complex128 else 1e-5)
    assert np.max(np.abs(n - n_ref) / n_ref) <= (1e-12 if dtype == np.complex128 else 1e-6)


@pytest.mark.parametrize("path", ["blk_real", "blk_cplx", "blk_64b", "blk_2cta"])
@pytest.mark.parametrize("zb", [0, 5, 9])
def test_blk_zblocks_and_tiles(cuda, monkeypatch, zb, path):
    """A box several tiles wide in x and y, cut into z blocks of several depths
    (the block edges re-read a 4-plane halo)."""
    import torch
    from hpsi import fixtures, lib
    from hpsi.mesh import index_box_mesh
    _set_path(monkeypatch, path, zb=zb)
    rng = np.random.default_rng(43)
    m = index_box_mesh((37, 21, 19), 0.3)
    v = fixtures.soft_coulomb(m, rng)
    psi = fixtures.random_states(m, 16, rng, orthonormal=False)
    dm, ham, w, pts = _setup(m, v=v)
    ref = _oracle(m, w, pts, v=v).apply(psi)
    x = _dev(psi, cuda, 16, np.complex128)
    y = torch.zeros((m.np, 16), dtype=x.dtype, device=cuda)
    ham.apply(x, y)
    assert rel_maxnorm_per_state(y.cpu().numpy(), ref) <= TOL64


@pytest.mark.parametrize("path", ["blk_real", "blk_cplx", "blk_64b", "blk_2cta"])
def test_blk_periodic_and_raw_boundary(cuda, monkeypatch, path):
    """Periodic images without Bloch phase (map to inner rows) and set_bc=False
    (boundary rows read as stored: the input tensor spans np_part rows)."""
    import torch
    from hpsi import fixtures, lib
    from hpsi.mesh import index_box_mesh, sphere_mesh
    _set_path(monkeypatch, path)
    rng = np.random.default_rng(47)
    m = index_box_mesh((12, 10, 8), 0.3, periodic=True)
    v = fixtures.soft_coulomb(m, rng)
    psi = fixtures.random_states(m, 8, rng, orthonormal=False)
    dm, ham, w, pts = _setup(m, v=v)
    ref = _oracle(m, w, pts, v=v, bc="periodic").apply(psi)
    x = _dev(psi, cuda, 8, np.complex128)
    y = torch.zeros((m.np, 8), dtype=x.dtype, device=cuda)
    ham.apply(x, y)
    assert rel_maxnorm_per_state(y.cpu().numpy(), ref) <= TOL64

    m = sphere_mesh(3.0, 0.4)
    r2 = np.sum(m.x * m.x, axis=1)
    f = (10 * np.exp(0.345j) * np.exp(-(1 / 3.0 + 0.01j) * r2) + (100 - 50j))[:, None] * \
        np.exp(0.1j * np.arange(8))[None, :]
    dm, ham, w, pts = _setup(m)
    ref = _oracle(m, w, pts, bc="none").apply(f)
    xd = _dev(f, cuda, 8, np.complex128)
    y = torch.zeros((m.np, 8), dtype=torch.complex128, device=cuda)
    ham.apply(xd, y, terms=1, set_bc=False)
    assert rel_maxnorm_per_state(y.cpu().numpy(), ref) <= TOL64


def test_paths_agree_fp32(cuda, monkeypatch):
    """The two FP32 kernels sum in different orders; they agree to FP32 rounding."""
    import torch
    m, v, proj, psi = small_sphere_system(seed=53, nst=16, radius=4.2, natoms=4)
    outs = []
    for path in PATHS:
        _set_path(monkeypatch, path)
        dm, ham, w, pts = _setup(m, v=v, proj=proj)
        x = _dev(psi, cuda, 16, np.complex64)
        y = torch.zeros((m.np, 16), dtype=x.dtype, device=cuda)
        ham.apply(x, y)
        outs.append(y.cpu().numpy().astype(np.complex128))
    for o in outs[1:]:
        assert rel_maxnorm_per_state(o, outs[0]) <= 2e-6


@pytest.mark.parametrize("dtype,ld", [(np.complex128, 32), (np.complex64, 64), (np.complex128, 12),
                                      (np.complex128, 64), (np.complex64, 128)])
@pytest.mark.parametrize("set_bc", [True, False])
def test_host_batches_pipelined(cuda, dtype, ld, set_bc):
    """Host (pinned) batches go through the slab pipeline (copy-in, passes,
    copy-out on three streams) when the width splits into chunk-aligned slabs,
    else through one staged pass; both equal the device-resident result."""
    import torch
    m, v, proj, psi = small_sphere_system(seed=59, nst=ld, radius=4.2, natoms=4)
    dm, ham, w, pts = _setup(m, v=v, proj=proj)
    x = _dev(psi, cuda, ld, dtype)
    y = torch.zeros((m.np, ld), dtype=x.dtype, device=cuda)
    ham.apply(x, y, set_bc=set_bc)
    xh = x.cpu().pin_memory()
    yh = torch.zeros((m.np, ld), dtype=x.dtype).pin_memory()
    ham.apply(xh, yh, set_bc=set_bc)
    # slabs change the projector split-K sums (rounding only)
    tol = 1e-13 if dtype == np.complex128 else 1e-6
    assert rel_maxnorm_per_state(yh.numpy().astype(np.complex128), y.cpu().numpy().astype(np.complex128)) <= tol


@pytest.mark.parametrize("dtype,ld", [(np.complex128, 3), (np.complex64, 6), (np.complex64, 10), (np.complex128, 40)])
def test_projector_bra_widths(cuda, dtype, ld):
    """KB bra on the FP64 tensor cores for any batch width (lanes past the
    width zero-filled; FP32 rows are 16-byte aligned only for even widths,
    which the library requires)."""
    import torch
    m, v, proj, psi = small_sphere_system(seed=61, nst=ld, radius=4.2, natoms=4)
    dm, ham, w, pts = _setup(m, v=v, proj=proj)
    ref = _oracle(m, w, pts, v=v, proj=proj).apply(psi)
    x = _dev(psi, cuda, ld, dtype)
    y = torch.zeros((m.np, ld), dtype=x.dtype, device=cuda)
    ham.apply(x, y)
    tol = TOL64 if dtype == np.complex128 else TOL32
    assert rel_maxnorm_per_state(y.cpu().numpy().astype(np.complex128), ref) <= tol


def test_odd_fp32_width_rejected(cuda):
    import torch
    from hpsi import lib
    m, v, proj, psi = small_sphere_system(seed=61, nst=5, radius=3.6, natoms=2)
    dm, ham, w, pts = _setup(m, v=v, proj=proj)
    x = _dev(psi, cuda, 5, np.complex64)
    y = torch.zeros((m.np, 5), dtype=x.dtype, device=cuda)
    with pytest.raises(lib.HpsiError, match="16-byte"):
        ham.apply(x, y)


@pytest.mark.parametrize("path", ["default", "blk_real", "blk_cplx", "blk_64b", "blk_2cta"])
@pytest.mark.parametrize("dtype,ld", [(np.complex128, 8), (np.complex64, 16)])
def test_blk_bloch_phase(cuda, monkeypatch, path, dtype, ld):
    """Bloch-phase periodic images (phase multiplied on load) in the blocked pass."""
    import torch
    from hpsi import fixtures
    from hpsi.mesh import index_box_mesh
    _set_path(monkeypatch, path)
    rng = np.random.default_rng(67)
    m = index_box_mesh((12, 10, 8), 0.3, periodic=True)
    v = fixtures.soft_coulomb(m, rng)
    psi = fixtures.random_states(m, ld, rng, orthonormal=False)
    k = np.array([0.3, -0.2, 0.5])
    pc = np.exp(1j * ((m.x[m.np:] - m.x[m.per_inner]) @ k))
    dm, ham, w, pts = _setup(m, v=v)
    ham.set_phase_corr(pc)
    from oracle import oracle as O
    ref = O.Hamiltonian(m, w, pts, v=v, bc="periodic", phase_corr=pc).apply(psi)
    x = _dev(psi, cuda, ld, dtype)
    y = torch.zeros((m.np, ld), dtype=x.dtype, device=cuda)
    ham.apply(x, y)
    tol = TOL64 if dtype == np.complex128 else TOL32
    assert rel_maxnorm_per_state(y.cpu().numpy().astype(np.complex128), ref) <= tol
