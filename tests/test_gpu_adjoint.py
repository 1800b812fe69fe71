"""Adjoint gradient of the Taylor propagator: the oracle's forward
propagation, central finite differences, the continuous-adjoint (reference
opt_control) gradient, and a torch.autograd.Function wrapper used as a harness."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(cuda, nsteps=30, nst=4, seed=11):
    import torch
    from hpsi import fixtures, lib
    from hpsi.mesh import index_box_mesh
    from hpsi.stencil import laplacian_weights, star_points
    rng = np.random.default_rng(seed)
    m = index_box_mesh((10, 9, 8), 0.3)
    v = fixtures.soft_coulomb(m, rng)
    psi = fixtures.random_states(m, nst, rng)
    phi = fixtures.random_states(m, nst, rng)
    eps = rng.normal(0.0, 0.05, size=nsteps)
    dm = lib.DeviceMesh(m)
    ham = lib.Hamiltonian(dm, laplacian_weights(m.spacing), star_points(), v=v)
    x = torch.from_numpy(psi).to(cuda)
    t = torch.from_numpy(phi).to(cuda)
    return m, v, psi, phi, eps, dm, ham, x, t


def test_adjoint_forward_matches_oracle(cuda):
    from oracle import oracle as O
    from hpsi.stencil import laplacian_weights, star_points
    m, v, psi, phi, eps, dm, ham, x, t = _setup(cuda)
    J, ge, gv, gc = ham.adjoint_gradient(x, t, eps, 0.02, ckpt=7)
    H = O.Hamiltonian(m, laplacian_weights(m.spacing), star_points(), v=v.copy())
    z = m.x[: m.np, 2]
    y = psi.copy()
    for e in eps:
        H.v[:] = v + e * z
        r = H.taylor(y, 0.02)
        y = np.zeros_like(y)
        y[: m.np] = r
    ov = m.vol_pp * np.sum(phi[: m.np].conj() * y[: m.np], axis=0)
    Jr = float(np.sum(np.abs(ov) ** 2))
    assert abs(J - Jr) <= 1e-12 * abs(Jr)
    assert np.array_equal(x.cpu().numpy(), psi)  # the input batch is untouched


@pytest.mark.parametrize("nst", [4, 12])
def test_adjoint_gradients_match_finite_differences(cuda, nst):
    """4 states: four mesh rows per warp in the gradient accumulation; 12
    states: two rows per warp."""
    m, v, psi, phi, eps, dm, ham, x, t = _setup(cuda, nst=nst)
    J, ge, gv, gc = ham.adjoint_gradient(x, t, eps, 0.02, ckpt=7)
    rng = np.random.default_rng(3)
    h = 1e-4
    for k in rng.choice(len(eps), 5, replace=False):
        ep, em = eps.copy(), eps.copy()
        ep[k] += h
        em[k] -= h
        fd = (ham.adjoint_gradient(x, t, ep, 0.02, want_v=False)[0] -
              ham.adjoint_gradient(x, t, em, 0.02, want_v=False)[0]) / (2 * h)
        assert abs(fd - ge[k]) <= 1e-6 * max(abs(ge[k]), 1e-3 * np.max(np.abs(ge)))
    hv = 1e-4
    for r in rng.choice(m.np, 5, replace=False):
        vp, vm = v.copy(), v.copy()
        vp[r] += hv
        vm[r] -= hv
        ham.set_vloc(vp)
        Jp = ham.adjoint_gradient(x, t, eps, 0.02, want_v=False)[0]
        ham.set_vloc(vm)
        Jm = ham.adjoint_gradient(x, t, eps, 0.02, want_v=False)[0]
        ham.set_vloc(v)
        fd = (Jp - Jm) / (2 * hv)
        assert abs(fd - gv[r]) <= 1e-6 * max(abs(gv[r]), 1e-3 * np.max(np.abs(gv)))


def test_checkpoint_interval_does_not_change_result(cuda):
    m, v, psi, phi, eps, dm, ham, x, t = _setup(cuda)
    a = ham.adjoint_gradient(x, t, eps, 0.02, ckpt=1)
    b = ham.adjoint_gradient(x, t, eps, 0.02, ckpt=30)
    assert a[0] == b[0]
    assert np.max(np.abs(a[1] - b[1])) <= 1e-14 * np.max(np.abs(a[1]))


def test_continuous_adjoint_gradient_agrees_in_direction(cuda):
    """The reference's 2 dt Im<chi|z|psi> is the leading term of the exact one."""
    m, v, psi, phi, eps, dm, ham, x, t = _setup(cuda)
    J, ge, gv, gc = ham.adjoint_gradient(x, t, eps, 0.02)
    cos = float(ge @ gc / (np.linalg.norm(ge) * np.linalg.norm(gc)))
    assert cos >= 0.95
    assert np.linalg.norm(ge - gc) <= 0.5 * np.linalg.norm(ge)


def test_torch_autograd_wrapper(cuda):
    import torch
    m, v, psi, phi, eps, dm, ham, x, t = _setup(cuda)

    class TaylorControl(torch.autograd.Function):
        @staticmethod
        def forward(ctx, e):
            J, ge, _, _ = ham.adjoint_gradient(x, t, e.detach().cpu().numpy(), 0.02, want_v=False)
            ctx.save_for_backward(torch.from_numpy(ge))
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            (ge,) = ctx.saved_tensors
            return gout * ge

    e = torch.tensor(eps, dtype=torch.float64, requires_grad=True)
    J = TaylorControl.apply(e)
    (g,) = torch.autograd.grad(J, e)
    _, ge, _, _ = ham.adjoint_gradient(x, t, eps, 0.02, want_v=False)
    assert np.array_equal(g.numpy(), ge)


def test_per_step_adjoint_equals_gradient(cuda):
    """A host-driven backward run (the shape of the reference's bwd_step loop):
    forward steps with hpsi_taylor_step under the field eps_n z, lambda_N from
    the target overlaps, then hpsi_adjoint_step for n = N-1 .. 0.  The per-step
    VJPs equal hpsi_adjoint_gradient (checkpointed, recomputing) to 1e-13."""
    import torch
    nsteps, dt = 12, 0.02
    m, v, psi, phi, eps, dm, ham, x, t = _setup(cuda, nsteps=nsteps)
    J, ge_ref, gv_ref, gc_ref = ham.adjoint_gradient(x, t, eps, dt, ckpt=5)
    xs = [x.clone()]
    cur = x.clone()
    for n in range(nsteps):
        ham.set_field((0.0, 0.0, 1.0), eps[n])
        ham.taylor_step(cur, dt)
        xs.append(cur.clone())
    ham.set_field((0.0, 0.0, 1.0), 0.0)
    yN = xs[-1][: m.np].cpu().numpy()
    ov = m.vol_pp * np.sum(phi[: m.np].conj() * yN, axis=0)
    assert abs(float(np.sum(np.abs(ov) ** 2)) - J) <= 1e-12 * J
    lam = torch.zeros_like(x)
    lam[: m.np] = torch.from_numpy(phi[: m.np] * ov[None, :]).to(cuda)
    gv = torch.zeros(m.np, dtype=torch.float64, device=cuda)
    ge, gc = np.zeros(nsteps), np.zeros(nsteps)
    for n in range(nsteps - 1, -1, -1):
        ge[n], gc[n] = ham.adjoint_step(lam, xs[n], eps[n], dt, grad_v=gv)
    assert np.max(np.abs(ge - ge_ref)) <= 1e-13 * np.max(np.abs(ge_ref))
    assert np.max(np.abs(gc - gc_ref)) <= 1e-13 * np.max(np.abs(gc_ref))
    gvh = gv.cpu().numpy()
    assert np.max(np.abs(gvh - gv_ref)) <= 1e-13 * np.max(np.abs(gv_ref))
    # the continuous-adjoint term is the reference's 2 dt Im <lambda|z|psi_n>:
    # one call of the field VJP on the same pair gives it
    lam_n1 = torch.zeros_like(x)
    lam_n1[: m.np] = torch.from_numpy(phi[: m.np] * ov[None, :]).to(cuda)
    d = ham.vjp_field(lam_n1, xs[nsteps - 1])
    assert abs(2 * dt * np.sum(d).imag - gc[nsteps - 1]) <= 1e-13 * abs(gc[nsteps - 1]) + 1e-18


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_vjp_field_and_vloc_match_numpy(cuda, dtype):
    import torch
    from hpsi import lib
    from hpsi.mesh import index_box_mesh
    from hpsi.stencil import laplacian_weights, star_points
    rng = np.random.default_rng(17)
    m = index_box_mesh((11, 9, 7), 0.3)
    nst = 37  # more states than a warp
    cdt = np.complex128 if dtype == "c128" else np.complex64
    a = (rng.standard_normal((m.np_part, nst)) + 1j * rng.standard_normal((m.np_part, nst))).astype(cdt)
    b = (rng.standard_normal((m.np_part, nst)) + 1j * rng.standard_normal((m.np_part, nst))).astype(cdt)
    ham = lib.Hamiltonian(lib.DeviceMesh(m), laplacian_weights(m.spacing), star_points())
    ta, tb = torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda)
    pol = np.array([0.3, -0.5, 0.8])
    z = m.x[: m.np] @ pol
    A, Bm = a[: m.np].astype(np.complex128), b[: m.np].astype(np.complex128)
    ref = m.vol_pp * np.sum(A.conj() * z[:, None] * Bm, axis=0)
    got = ham.vjp_field(ta, tb, pol=pol)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    g = torch.full((m.np,), 7.0, dtype=torch.float64, device=cuda)
    ham.vjp_vloc(ta, tb, g, scale=0.25)
    refv = 0.25 * np.sum((A.conj() * Bm).real, axis=1)
    assert np.max(np.abs(g.cpu().numpy() - refv)) <= 1e-12 * np.max(np.abs(refv))
    ham.vjp_vloc(ta, tb, g, scale=0.25, accumulate=True)
    assert np.max(np.abs(g.cpu().numpy() - 2 * refv)) <= 1e-12 * np.max(np.abs(refv))
