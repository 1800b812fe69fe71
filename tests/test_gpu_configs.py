"""GPU parity at the full sizes of the benchmark configurations.

The small-mesh parity tests cover every code path on shapes the oracle
finishes in milliseconds; these run the two configurations the bench measures
at their real sizes, where the work lists have thousands of items, the
split-K bra sums many partial blocks and every state chunk of a 128-wide batch
is in flight:

* sphere R = 12 bohr, h = 0.2 (904,089 inner points), 32 KB atoms x 9
  projectors, 128 complex128 states (the headline H psi);
* box 64^3, h = 0.25, 32 states, kinetic + local.

The device computes the whole batch; the oracle (FP64 CPU, the reference's
compiled stencil) computes a sample of states spread over the state chunks,
and each sampled state is compared by the parity metric (relative max-norm
per state): FP64 <= 1e-12, FP32 storage <= 2e-5.  Size-independent checks
run on the whole batch: the Hermiticity of H on the sampled pairs and the
norm change of one Taylor step.
"""
import numpy as np
import pytest

from helpers import rel_maxnorm_per_state

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5
SAMPLE1 = [0, 17, 38, 63, 64, 90, 111, 127]  # states of the 128-wide batch
SAMPLE0 = [0, 9, 22, 31]


class _Sys:
    pass


def _build(cfg, cuda):
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O
    s = _Sys()
    s.cfg = cfg
    m = cfg.mesh
    w = laplacian_weights(m.spacing)
    s.dm = lib.DeviceMesh(m)
    s.ham = lib.Hamiltonian(s.dm, w, star_points(), v=cfg.v, projectors=cfg.proj)
    P = None if cfg.proj is None else O.Projectors(cfg.proj.maps, cfg.proj.mats, cfg.proj.scals)
    s.oracle = O.Hamiltonian(m, w, star_points(), v=cfg.v, projectors=P)
    s.x = torch.from_numpy(cfg.psi).to(cuda)
    return s


@pytest.fixture(scope="module")
def sphere128(cuda):
    from hpsi import fixtures
    return _build(fixtures.config1(), cuda)


@pytest.fixture(scope="module")
def box64(cuda):
    from hpsi import fixtures
    return _build(fixtures.config0(), cuda)


def _check_apply(s, sample, dtype, tol):
    import torch
    m = s.cfg.mesh
    nst = s.cfg.psi.shape[1]
    x = s.x if dtype == torch.complex128 else s.x.to(dtype)
    y = torch.zeros((m.np, nst), dtype=dtype, device=x.device)
    s.ham.apply(x, y)
    got = y[:, sample].cpu().numpy().astype(np.complex128)
    ref = s.oracle.apply(np.ascontiguousarray(s.cfg.psi[:, sample]))
    err = rel_maxnorm_per_state(got, ref)
    assert err <= tol, f"relative max-norm {err:.3e}"
    return y


def _check_taylor(s, sample, dtype, tol, dt):
    import torch
    m = s.cfg.mesh
    x = s.x.clone() if dtype == torch.complex128 else s.x.to(dtype)
    n0 = s.dm.nrm2(x)
    s.ham.taylor_step(x, dt)
    got = x[: m.np, sample].cpu().numpy().astype(np.complex128)
    ref = s.oracle.taylor(np.ascontiguousarray(s.cfg.psi[:, sample]), dt)
    err = rel_maxnorm_per_state(got, ref)
    assert err <= tol, f"relative max-norm {err:.3e}"
    # whole batch: the norm change of every state (the truncated series is
    # not unitary at these dt) stays of the size the oracle shows for the
    # sampled states, statistically alike
    n1 = s.dm.nrm2(x)
    ch = np.abs(n1 - n0) / n0
    ref_ch = np.abs(np.sqrt(np.sum(np.abs(ref) ** 2, axis=0) * m.vol_pp) - n0[sample]) / n0[sample]
    assert np.all(np.isfinite(n1))
    assert np.max(np.abs(ch[sample] - ref_ch)) <= (1e-12 if dtype == torch.complex128 else 1e-5)
    assert np.max(ch) <= 10.0 * np.max(ref_ch) + 1e-12


def test_sphere128_hpsi_fp64(sphere128):
    import torch
    y = _check_apply(sphere128, SAMPLE1, torch.complex128, TOL64)
    # H is Hermitian on the inner points: <a|H b> = conj(<b|H a>) for sampled
    # pairs (the zero boundary holds the whole batch to the same operator)
    m = sphere128.cfg.mesh
    a, b = SAMPLE1[1], SAMPLE1[-2]
    xa = sphere128.x[: m.np, a]
    xb = sphere128.x[: m.np, b]
    lhs = torch.vdot(xa, y[:, b]).item()
    rhs = np.conj(torch.vdot(xb, y[:, a]).item())
    # Cauchy-Schwarz bound of the summed terms: the scale of the rounding
    scale = (xa.norm() * y[:, b].norm() + xb.norm() * y[:, a].norm()).item()
    assert abs(lhs - rhs) <= 1e-12 * scale


def test_sphere128_hpsi_fp32(sphere128):
    import torch
    _check_apply(sphere128, SAMPLE1, torch.complex64, TOL32)


def test_sphere128_taylor_fp64(sphere128):
    import torch
    _check_taylor(sphere128, SAMPLE1, torch.complex128, TOL64, 0.005)


def test_sphere128_taylor_fp32(sphere128):
    import torch
    _check_taylor(sphere128, SAMPLE1, torch.complex64, TOL32, 0.005)


def test_box64_hpsi_fp64(box64):
    import torch
    _check_apply(box64, SAMPLE0, torch.complex128, TOL64)


def test_box64_hpsi_fp32(box64):
    import torch
    _check_apply(box64, SAMPLE0, torch.complex64, TOL32)


def test_box64_taylor_fp64(box64):
    import torch
    _check_taylor(box64, SAMPLE0, torch.complex128, TOL64, 0.01)


def test_box64_taylor_fp32(box64):
    import torch
    _check_taylor(box64, SAMPLE0, torch.complex64, TOL32, 0.01)


def test_sphere128_hpsi_linearity(sphere128):
    """Linearity of the full-size H psi over the whole 128-state batch:
    H(x1 + c x2) = H x1 + c H x2 for x2 the batch with its states rotated and
    a complex c, every state compared (not only the oracle's sample)."""
    import torch
    s = sphere128
    m = s.cfg.mesh
    x1 = s.x
    x2 = torch.roll(s.x, shifts=37, dims=1)
    c = 0.3 - 0.7j
    y1 = torch.zeros((m.np, x1.shape[1]), dtype=x1.dtype, device=x1.device)
    y2 = torch.zeros_like(y1)
    y3 = torch.zeros_like(y1)
    s.ham.apply(x1, y1)
    s.ham.apply(x2, y2)
    s.ham.apply(x1 + c * x2, y3)
    ref = (y1 + c * y2).cpu().numpy()
    assert rel_maxnorm_per_state(y3.cpu().numpy(), ref) <= 1e-13


def test_config3_group_at_full_size(cuda):
    """Eight of the uneven systems of the grouped configuration at their real
    sizes (boxes of 32 to 95 cells a side, 4 to 58 states, KB atoms): two
    grouped Taylor steps (one persistent launch per pass, CUDA graph) against
    the same systems propagated one by one."""
    import torch
    from hpsi import fixtures, lib
    from hpsi.stencil import laplacian_weights, star_points
    systems = fixtures.config3(nsys=64)[:8]
    keep, xs, refs = [], [], []
    for sy in systems:
        dm = lib.DeviceMesh(sy.mesh)
        h = lib.Hamiltonian(dm, laplacian_weights(sy.mesh.spacing), star_points(), v=sy.v, projectors=sy.proj)
        x = torch.from_numpy(sy.psi).to(cuda)
        r = x.clone()
        for _ in range(2):
            h.taylor_step(r, 0.01)
        keep.append((dm, h))
        xs.append(x)
        refs.append(r)
    g = lib.Group([h for _, h in keep])
    g.taylor_steps(xs, 2, 0.01)
    for sy, x, r in zip(systems, xs, refs):
        n = sy.mesh.np
        assert rel_maxnorm_per_state(x[:n].cpu().numpy(), r[:n].cpu().numpy()) <= 1e-13
    g.close()


def test_config4_adjoint_gradient_full_size(cuda):
    """The adjoint configuration at its real size (64^3 box, h = 0.25, 16
    states, 500 steps, checkpoints every 25): the gradient with respect to
    three control amplitudes against central finite differences of J."""
    import torch
    from hpsi import fixtures, lib
    from hpsi.stencil import laplacian_weights, star_points
    s0 = fixtures.config0(nst=16)
    m = s0.mesh
    dm = lib.DeviceMesh(m)
    ham = lib.Hamiltonian(dm, laplacian_weights(m.spacing), star_points(), v=s0.v)
    eps = np.random.default_rng(7).normal(0.0, 0.005, 500)
    psi0 = torch.from_numpy(s0.psi).to(cuda)
    tg = torch.from_numpy(fixtures.random_states(m, 16, np.random.default_rng(8))).to(cuda)
    J, ge, gv, gc = ham.adjoint_gradient(psi0, tg, eps, 0.01, ckpt=25, want_v=False)
    assert np.all(np.isfinite(ge))
    h = 1e-4
    for k in (3, 250, 497):
        ep, em = eps.copy(), eps.copy()
        ep[k] += h
        em[k] -= h
        jp = ham.adjoint_gradient(psi0, tg, ep, 0.01, ckpt=25, want_v=False)[0]
        jm = ham.adjoint_gradient(psi0, tg, em, 0.01, ckpt=25, want_v=False)[0]
        fd = (jp - jm) / (2 * h)
        assert abs(fd - ge[k]) <= 1e-5 * np.max(np.abs(ge)), (k, fd, ge[k])
