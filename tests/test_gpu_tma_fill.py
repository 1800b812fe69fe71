"""Variants of the blocked stencil pass that move the same data by other
means, checked bit for bit against the default (per-thread cp.async fill, one
barrier per plane):

* TMA fill: runs of eight consecutive batch rows in a halo row arrive as one
  cp.async.bulk.tensor box (8 rows x 128 bytes) completing on the stage's
  mbarrier; the other halo cells keep their per-thread copies;
* mbarrier hand-over: the per-thread fill, with each stage handed over by a
  full and an empty mbarrier (cp.async arrive-on) instead of the barrier.

The same values land in shared memory and are summed in the same order, so
H psi, a Taylor step (with and without the observables of its first pass)
equal the default bit for bit (zero boundary map, raw map with set_bc = 0, a
KB system, FP64 and FP32), and the Hamiltonian's status word stays clear (no
bounded wait gave up)."""
import numpy as np
import pytest

from helpers import small_sphere_system

pytestmark = pytest.mark.gpu

SHAPES = {
    "tma": {"c128": ("HPSI_PASS_SHAPE64", "8,2,0,9,1,2,0,8,1"), "c64": ("HPSI_PASS_SHAPE32", "16,2,0,9,1,2,1,8,1")},
    "mbar": {"c128": ("HPSI_PASS_SHAPE64", "8,2,0,9,1,2,0,8,0,1"),
             "c64": ("HPSI_PASS_SHAPE32", "16,2,0,9,1,2,1,8,0,1")},
}


@pytest.mark.parametrize("variant", ["tma", "mbar"])
@pytest.mark.parametrize("dtype,nst", [("c128", 16), ("c64", 32)])
def test_fill_variant_equals_default_fill(cuda, dtype, nst, variant, monkeypatch):
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    var, shape = SHAPES[variant][dtype]
    m, v, proj, psi = small_sphere_system(seed=83, nst=nst, radius=4.5, natoms=3)
    H = lib.Hamiltonian(lib.DeviceMesh(m), laplacian_weights(m.spacing), star_points(), v=v, projectors=proj)
    x = torch.from_numpy(psi).to(cuda).to(tdt)

    def run():
        ya = torch.zeros((m.np, nst), dtype=tdt, device=cuda)
        H.apply(x, ya)
        yr = torch.zeros_like(ya)
        H.apply(x, yr, set_bc=False)
        xt = x.clone()
        H.taylor_step(xt, 0.01)
        xo = x.clone()
        obs = H.taylor_step(xo, 0.01, observables=True)
        return (ya, yr, xt, xo), obs

    monkeypatch.delenv(var, raising=False)
    ref, ref_obs = run()
    monkeypatch.setenv(var, shape)
    got, got_obs = run()
    assert H.status() == 0
    for a, b in zip(ref, got):
        assert torch.equal(a, b)
    for a, b in zip(np.atleast_1d(ref_obs), np.atleast_1d(got_obs)):
        assert np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("variant", ["tma", "mbar"])
def test_fill_variant_box_mesh_default_order(cuda, variant, monkeypatch):
    """A box mesh (long runs of consecutive rows in the blocked point order:
    most of the halo arrives by TMA) at a width of several state chunks."""
    import torch
    from hpsi import fixtures, lib
    from hpsi.mesh import index_box_mesh
    from hpsi.stencil import laplacian_weights, star_points
    rng = np.random.default_rng(84)
    m = index_box_mesh((40, 36, 30), 0.25)
    v = fixtures.soft_coulomb(m, rng)
    psi = fixtures.random_states(m, 24, rng, orthonormal=False)
    H = lib.Hamiltonian(lib.DeviceMesh(m), laplacian_weights(m.spacing), star_points(), v=v)
    x = torch.from_numpy(psi).to(cuda)
    var, shape = SHAPES[variant]["c128"]
    monkeypatch.delenv(var, raising=False)
    y0 = torch.zeros((m.np, 24), dtype=torch.complex128, device=cuda)
    H.apply(x, y0)
    monkeypatch.setenv(var, shape)
    y1 = torch.zeros_like(y0)
    H.apply(x, y1)
    assert H.status() == 0
    assert torch.equal(y0, y1)
