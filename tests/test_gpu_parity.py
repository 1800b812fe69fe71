"""GPU parity: the CUDA path through the C ABI against the FP64 CPU oracle.

Gate (FP64): relative max-norm per state <= 1e-12.  FP32-storage forms are
checked against the same oracle at 2e-5 (single-precision rounding).
"""
import numpy as np
import pytest

from helpers import rel_maxnorm_per_state, small_sphere_system

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def _setup(mesh, v=None, proj=None):
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    w = laplacian_weights(mesh.spacing)
    pts = star_points()
    dm = lib.DeviceMesh(mesh)
    ham = lib.Hamiltonian(dm, w, pts, v=v, projectors=proj)
    return dm, ham, w, pts


def _oracle(mesh, w, pts, v=None, proj=None, bc="zero", phase_corr=None):
    from oracle import oracle as O
    P = None
    if proj is not None:
        P = O.Projectors(proj.maps, proj.mats, proj.scals)
    return O.Hamiltonian(mesh, w, pts, v=v, projectors=P, bc=bc, phase_corr=phase_corr)


def _dev(x, cuda, ld=None, dtype=None):
    import torch
    x = np.asarray(x)
    ld = ld or x.shape[1]
    out = np.zeros((x.shape[0], ld), dtype=x.dtype if dtype is None else dtype)
    out[:, : x.shape[1]] = x
    return torch.from_numpy(out).to(cuda)


def test_apply_box_kinetic_local(cuda):
    import torch
    from hpsi import fixtures
    from hpsi.mesh import index_box_mesh
    rng = np.random.default_rng(0)
    m = index_box_mesh((13, 11, 9), 0.25)
    v = fixtures.soft_coulomb(m, rng)
    psi = fixtures.random_states(m, 5, rng)
    dm, ham, w, pts = _setup(m, v=v)
    ref = _oracle(m, w, pts, v=v).apply(psi)
    x = _dev(psi, cuda, ld=8)
    y = torch.zeros((m.np, 8), dtype=torch.complex128, device=cuda)
    ham.apply(x, y, nst=5)
    torch.cuda.synchronize()
    got = y.cpu().numpy()[:, :5]
    assert rel_maxnorm_per_state(got, ref) <= TOL64


def test_apply_sphere_kb_all_terms(cuda):
    import torch
    m, v, proj, psi = small_sphere_system()
    dm, ham, w, pts = _setup(m, v=v, proj=proj)
    ref = _oracle(m, w, pts, v=v, proj=proj).apply(psi)
    x = _dev(psi, cuda, ld=8)
    y = torch.zeros((m.np, 8), dtype=torch.complex128, device=cuda)
    ham.apply(x, y, nst=psi.shape[1])
    got = y.cpu().numpy()[:, : psi.shape[1]]
    assert rel_maxnorm_per_state(got, ref) <= TOL64


@pytest.mark.parametrize("terms", [1, 2, 4, 3, 5, 6])
def test_apply_terms(cuda, terms):
    import torch
    from oracle import oracle as O
    m, v, proj, psi = small_sphere_system(seed=5, nst=4)
    dm, ham, w, pts = _setup(m, v=v, proj=proj)
    wk = w if terms & 1 else np.zeros_like(w)
    vv = v if terms & 2 else None
    pp = O.Projectors(proj.maps, proj.mats, proj.scals) if terms & 4 else None
    ref = O.Hamiltonian(m, wk, pts, v=vv, projectors=pp).apply(psi)
    x = _dev(psi, cuda)
    y = torch.zeros((m.np, 4), dtype=torch.complex128, device=cuda)
    ham.apply(x, y, terms=terms)
    got = y.cpu().numpy()
    scale = max(np.max(np.abs(ref)), 1e-300)
    assert np.max(np.abs(got - ref)) / scale <= TOL64


def test_point_order_independent(cuda):
    import torch
    from hpsi.mesh import permuted
    m, v, proj, psi = small_sphere_system(seed=7, nst=3)
    m2, perm, inv = permuted(m, seed=1)
    dm, ham, w, pts = _setup(m, v=v, proj=proj)
    proj2 = type(proj)([inv[mp].astype(np.int32) for mp in proj.maps], proj.mats, proj.scals, proj.positions)
    dm2, ham2, _, _ = _setup(m2, v=v[perm[: m.np]], proj=proj2)
    x = _dev(psi, cuda, ld=4)
    x2 = _dev(psi[perm], cuda, ld=4)
    y = torch.zeros((m.np, 4), dtype=torch.complex128, device=cuda)
    y2 = torch.zeros_like(y)
    ham.apply(x, y, nst=3)
    ham2.apply(x2, y2, nst=3)
    a = y.cpu().numpy()[:, :3]
    b = y2.cpu().numpy()[:, :3][inv[: m.np]]
    assert rel_maxnorm_per_state(b, a) <= TOL64


def test_periodic_bloch_phase(cuda):
    import torch
    from hpsi import fixtures
    from hpsi.mesh import index_box_mesh
    rng = np.random.default_rng(11)
    m = index_box_mesh((12, 10, 8), 0.3, periodic=True)
    v = fixtures.soft_coulomb(m, rng)
    psi = fixtures.random_states(m, 4, rng, orthonormal=False)
    k = np.array([0.3, -0.2, 0.5])
    # phase correction of each boundary point relative to its image
    dx = (m.x[m.np:] - m.x[m.per_inner]) @ k
    pc = np.exp(1j * dx)
    dm, ham, w, pts = _setup(m, v=v)
    ham.set_phase_corr(pc)
    ref = _oracle(m, w, pts, v=v, bc="periodic", phase_corr=pc).apply(psi)
    x = _dev(psi, cuda)
    y = torch.zeros((m.np, 4), dtype=torch.complex128, device=cuda)
    ham.apply(x, y)
    assert rel_maxnorm_per_state(y.cpu().numpy(), ref) <= TOL64
    # boundaries_set writes the same boundary rows as the oracle
    from oracle import oracle as O
    hb = _oracle(m, w, pts, v=v, bc="periodic", phase_corr=pc)
    xb, ld = O.Hamiltonian.packed(psi)
    import ctypes as C
    c = hb._ctx(ld, 4)
    O.lib().orc_boundaries_set(C.byref(c), O._p(xb.view(np.float64)))
    ham.boundaries_set(x)
    assert np.max(np.abs(x.cpu().numpy() - xb)) <= 1e-15 * np.max(np.abs(xb))


def test_set_bc_false_uses_stored_boundary(cuda):
    import torch
    from hpsi.mesh import sphere_mesh
    m = sphere_mesh(3.0, 0.4)
    x = m.x
    r2 = np.sum(x * x, axis=1)
    a, b, c = 1 / 3.0 + 0.01j, 10 * np.exp(0.345j), 100 - 50j
    f = (b * np.exp(-a * r2) + c)[:, None] * np.array([[1.0, 0.5 - 0.25j]])
    dm, ham, w, pts = _setup(m)
    ref = _oracle(m, w, pts, bc="none").apply(f)
    xd = _dev(f, cuda)
    y = torch.zeros((m.np, 2), dtype=torch.complex128, device=cuda)
    ham.apply(xd, y, terms=1, set_bc=False)
    assert rel_maxnorm_per_state(y.cpu().numpy(), ref) <= TOL64


@pytest.mark.parametrize("order", [1, 2, 4])
def test_taylor_step_fp64(cuda, order):
    m, v, proj, psi = small_sphere_system(seed=13, nst=6)
    dm, ham, w, pts = _setup(m, v=v, proj=proj)
    ref = _oracle(m, w, pts, v=v, proj=proj).taylor(psi, 0.02, order=order)
    x = _dev(psi, cuda, ld=8)
    ham.taylor_step(x, 0.02, order=order, nst=6)
    got = x.cpu().numpy()[: m.np, :6]
    assert rel_maxnorm_per_state(got, ref) <= TOL64


def test_taylor_observables(cuda):
    m, v, proj, psi = small_sphere_system(seed=17, nst=5)
    dm, ham, w, pts = _setup(m, v=v, proj=proj)
    h = _oracle(m, w, pts, v=v, proj=proj).apply(psi)
    dv = m.vol_pp
    e_ref = dv * np.real(np.sum(psi[: m.np].conj() * h, axis=0))
    n_ref = dv * np.sum(np.abs(psi[: m.np]) ** 2, axis=0)
    d_ref = dv * np.sum(np.abs(psi[: m.np]) ** 2 * m.x[: m.np, 2:3], axis=0)
    x = _dev(psi, cuda, ld=8)
    e, d, n = ham.taylor_step(x, 0.02, order=4, nst=5, observables=True)
    assert np.max(np.abs(e - e_ref) / np.abs(e_ref)) <= 1e-12
    assert np.max(np.abs(n - n_ref) / n_ref) <= 1e-12
    assert np.max(np.abs(d - d_ref)) <= 1e-12 * np.max(np.abs(n_ref)) * 4


def test_fp32_storage(cuda):
    import torch
    m, v, proj, psi = small_sphere_system(seed=19, nst=8)
    dm, ham, w, pts = _setup(m, v=v, proj=proj)
    o = _oracle(m, w, pts, v=v, proj=proj)
    ref = o.apply(psi)
    x = _dev(psi.astype(np.complex64), cuda)
    y = torch.zeros((m.np, 8), dtype=torch.complex64, device=cuda)
    ham.apply(x, y)
    assert rel_maxnorm_per_state(y.cpu().numpy().astype(np.complex128), ref) <= TOL32
    ref_t = o.taylor(psi, 0.02, order=4)
    ham.taylor_step(x, 0.02, order=4)
    assert rel_maxnorm_per_state(x.cpu().numpy()[: m.np].astype(np.complex128), ref_t) <= TOL32


def test_host_pointer_batches(cuda):
    import torch
    m, v, proj, psi = small_sphere_system(seed=23, nst=4)
    dm, ham, w, pts = _setup(m, v=v, proj=proj)
    ref = _oracle(m, w, pts, v=v, proj=proj).apply(psi)
    xh = np.ascontiguousarray(psi)
    yh = np.zeros((m.np, 4), dtype=np.complex128)
    ham.apply(xh, yh)
    assert rel_maxnorm_per_state(yh, ref) <= TOL64
    ref_t = _oracle(m, w, pts, v=v, proj=proj).taylor(psi, 0.01, order=4)
    ham.taylor_step(xh, 0.01)
    assert rel_maxnorm_per_state(xh[: m.np], ref_t) <= TOL64


def test_reductions(cuda):
    from oracle import oracle as O
    m, v, proj, psi = small_sphere_system(seed=29, nst=6)
    rng = np.random.default_rng(3)
    a = psi * (1 + 0.1 * rng.standard_normal(psi.shape))
    dm = _setup(m)[0]
    x = _dev(a, cuda, ld=8)
    y = _dev(psi, cuda, ld=8)
    nrm = dm.nrm2(x, nst=6)
    assert np.max(np.abs(nrm - O.mesh_batch_nrm2(m, a)) / O.mesh_batch_nrm2(m, a)) <= 1e-13
    S = dm.dotp_matrix(x, y, nst=6)
    S_ref = O.mesh_batch_dotp_matrix(m, a, psi)
    assert np.max(np.abs(S - S_ref)) <= 1e-13 * np.max(np.abs(S_ref))
    dm.orthonormalize_cholesky(x, nst=6)
    got = x.cpu().numpy()[: m.np, :6]
    ref = O.cholesky_orthonormalize(m, a)[: m.np]
    assert rel_maxnorm_per_state(got, ref) <= 1e-11
    S2 = dm.dotp_matrix(x, x, nst=6)
    assert np.max(np.abs(S2 - np.eye(6))) <= 1e-12


def test_index_errors_reported(cuda):
    from hpsi import lib
    from hpsi.mesh import Mesh, index_box_mesh
    m = index_box_mesh((6, 6, 6), 0.3)
    # drop the boundary points: inner stencils leave the mesh
    bad = Mesh(lxyz=np.ascontiguousarray(m.lxyz[: m.np]), np=m.np, spacing=m.spacing)
    with pytest.raises(lib.HpsiError) as e:
        lib.DeviceMesh(bad)
    assert e.value.status == 2
    dm, ham, w, pts = _setup(m)
    proj_maps = [np.array([0, 1, m.np + 3], dtype=np.int32)]
    with pytest.raises(lib.HpsiError) as e:
        ham.set_projectors(proj_maps, [np.ones((3, 2))], [np.ones(2)])
    assert e.value.status == 2


def test_nonfinite_detected(cuda):
    m, v, proj, psi = small_sphere_system(seed=31, nst=2)
    from hpsi import lib
    dm, ham, w, pts = _setup(m, v=v)
    bad = psi.copy()
    bad[5, 1] = np.nan
    x = _dev(bad, cuda)
    with pytest.raises(lib.HpsiError) as e:
        ham.taylor_step(x, 0.02, observables=True)
    assert e.value.status == 3


def test_update_vloc_is_stream_ordered(cuda):
    """hpsi_hamiltonian_update_vloc on a side stream (host input, then a
    device tensor), each followed by H psi on the same stream with no host
    synchronisation between them, against the oracle with that potential."""
    import torch
    from hpsi import lib
    m, v, proj, psi = small_sphere_system(seed=91, nst=8)
    dm, ham, w, pts = _setup(m, v=None, proj=proj)
    x = torch.from_numpy(psi).to(cuda)
    st = torch.cuda.Stream()
    v2 = torch.from_numpy(2.0 * v - 0.5).to(cuda)
    outs = []
    with torch.cuda.stream(st):
        for vv in (v, v2):
            ham.update_vloc(vv, stream=st)
            y = torch.zeros((m.np, 8), dtype=torch.complex128, device=cuda)
            ham.apply(x, y, stream=st)
            outs.append(y)
    st.synchronize()
    for y, vv in zip(outs, (v, 2.0 * v - 0.5)):
        ref = _oracle(m, w, pts, v=vv, proj=proj).apply(psi)
        assert rel_maxnorm_per_state(y.cpu().numpy(), ref) <= TOL64
    with pytest.raises(lib.HpsiError):
        bad = v.copy()
        bad[3] = np.nan
        ham.update_vloc(bad)
