"""CPU tests of the oracle (no GPU): pinned against the reference's own kernel."""
import ctypes as C
import os

import numpy as np
import pytest

from helpers import rel_maxnorm_per_state, small_sphere_system

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "ref_operate.npz")


def _mesh_from(g, name):
    from hpsi.mesh import Mesh
    return Mesh(lxyz=g[f"{name}_lxyz"], np=int(g[f"{name}_np"]), spacing=g[f"{name}_spacing"])


@pytest.mark.parametrize("name", ["sphere", "box"])
def test_restated_stencil_matches_reference_kernel_golden(name):
    """orc_operate_ri (the restatement) reproduces the reference operate.c output."""
    from oracle import oracle as O
    from hpsi.stencil import star_points
    g = np.load(GOLDEN)
    m = _mesh_from(g, name)
    w = g[f"{name}_weights"]
    x = np.ascontiguousarray(g[f"{name}_in"])
    ref = g[f"{name}_out"]
    op = O.Operator(m, star_points())
    wre = np.ascontiguousarray(w * -0.5)
    fo = np.zeros_like(ref)
    O.lib().orc_operate_ri(C.byref(C.c_int(25)), O._p(wre), C.byref(C.c_int(op.nri)), O._p(op.ri, C.c_int),
                           O._p(op.imin, C.c_int), O._p(op.imax, C.c_int), O._p(x.view(np.float64)),
                           C.byref(C.c_int(3)), O._p(fo.view(np.float64)))
    assert rel_maxnorm_per_state(fo[:, :3], ref[:, :3]) <= 1e-15


def test_weights_file_of_stencil_golden():
    """Regression check only: the weights the stencil golden was computed with
    (an input of the reference-kernel run in make_golden.py) are still the ones
    the host solve returns.  The weights are pinned externally by the two
    tests below."""
    from hpsi.stencil import laplacian_weights
    g = np.load(GOLDEN)
    for name in ("sphere", "box"):
        w = laplacian_weights(g[f"{name}_spacing"])
        assert np.array_equal(w, g[f"{name}_weights"])


@pytest.mark.parametrize("h", [0.1, 0.2, 0.25, 0.4])
def test_weights_close_to_closed_form(h):
    """Solved weights agree with the order-8 central-difference coefficients
    (-205/72, 8/5, -1/5, 8/315, -1/560) / h^2 to the accuracy an FP64 solve of
    the fit has (measured deviation 2.3e-13 relative at h = 0.2)."""
    from hpsi.stencil import laplacian_weights, star_points
    w = laplacian_weights(h)
    arm = {1: 8 / 5, 2: -1 / 5, 3: 8 / 315, 4: -1 / 560}
    pts = star_points()
    for j, p in enumerate(pts):
        d = int(np.abs(p).max())
        expect = (3 * (-205 / 72) if d == 0 else arm[d]) / h ** 2
        assert abs(w[j] - expect) <= 1e-12 * abs(expect)


@pytest.mark.parametrize("h", [0.2, 0.4])
def test_weights_satisfy_the_fit_conditions(h):
    """The linear system the reference solves for the star Laplacian
    (derivatives_make_discretization, src/grid/derivatives.F90:586-609,
    639-757; polynomials of stencil_star, src/grid/stencil_star.F90:97-116):
    exact on 1 and on x_i^n for n = 1..8 along each axis, with right-hand side
    2 for x_i^2 and 0 otherwise."""
    from hpsi.stencil import laplacian_weights, star_points
    w = laplacian_weights(h)
    x = star_points().astype(np.float64) * h
    scale = np.sum(np.abs(w))
    assert abs(np.sum(w)) <= 1e-14 * scale
    for ax in range(3):
        for n in range(1, 9):
            lhs = np.sum(w * x[:, ax] ** n)
            rhs = 2.0 if n == 2 else 0.0
            assert abs(lhs - rhs) <= 1e-13 * np.sum(np.abs(w * x[:, ax] ** n)) + 1e-13


def _deriv_errors(radius, h):
    from oracle import oracle as O
    from hpsi.mesh import sphere_mesh
    from hpsi.stencil import laplacian_weights, star_points
    m = sphere_mesh(radius, h)
    m.extra["bbox_l"] = radius
    w = laplacian_weights(h)
    return (O.derivatives_test_error(m, w, star_points(), False, use_ref=False),
            O.derivatives_test_error(m, w, star_points(), True, use_ref=False))


def test_derivatives_test_reproduces_reference_kernel_value():
    """X(derivatives_test) (src/grid/derivatives_inc.F90:378-492) on its own
    mesh (03-derivatives_3d.01.inp: sphere R = 8, h = 0.4, aa = 1/8): the
    restated stencil gives the Laplacian error norm the reference's compiled
    operate.c gave (stored by make_golden.py)."""
    g = np.load(GOLDEN)
    er, ec = _deriv_errors(8.0, 0.4)
    # the norm is a small difference of O(100) values: rounding of the two
    # kernels (vectorised vs scalar FMA order) shows at ~1e-9 relative
    assert abs(er - float(g["deriv_real"])) <= 1e-8 * abs(er)
    assert abs(ec - float(g["deriv_complex"])) <= 1e-8 * abs(ec)


def test_derivatives_test_error_is_eighth_order():
    """The same test at h = 0.4 and h = 0.2: the error of the order-4 star
    falls by 2^8 (truncation error O(h^8)); a wrong weight or a lower order
    changes the ratio (order 3 would give 2^6)."""
    er1, ec1 = _deriv_errors(8.0, 0.4)
    er2, ec2 = _deriv_errors(8.0, 0.2)
    assert 200.0 <= er1 / er2 <= 320.0
    assert 200.0 <= ec1 / ec2 <= 320.0


def test_reference_golden_values_are_a_scaling_error():
    """Why the printed goldens of 03-derivatives_3d.test (1.1962559177E-03 real,
    1.2044354237E-03 complex, tolerance 3e-3) are not reproduced: they do not
    behave like the truncation error of a finite-difference Laplacian of
    f = b exp(-a r^2) + c on this mesh, but like a relative scaling error of
    the Laplacian, err = eps * ||lapl f||.  The complex/real ratio of the two
    goldens is a fingerprint that does not depend on the size of the error:
    the scaling model predicts it to 6e-4, the truncation error of the
    order-4 star (what the source computes) misses it by 2.5 %.  The implied
    eps = 3.7e-5 would be a grid spacing 1.85e-5 relative off the one the
    weights were solved for.  The reference's own tolerance (3e-3) exceeds
    the golden value, so the reference test accepts our 1.71e-5."""
    from hpsi.mesh import sphere_mesh
    gold_r, gold_c = 1.1962559177e-03, 1.2044354237e-03
    m = sphere_mesh(8.0, 0.4)
    x = m.x[: m.np]
    r2 = np.sum(x ** 2, axis=1)
    a, b = 1.0 / 8.0, 10.0

    def lapl_norm(aa, bb):
        L = bb * (4 * aa ** 2 * r2 - 6 * aa) * np.exp(-aa * r2)
        return np.sqrt(np.sum(np.abs(L) ** 2) * m.vol_pp)

    ratio_scaling = lapl_norm(a + 0.01j, b * np.exp(0.345j)) / lapl_norm(a, b)
    er, ec = _deriv_errors(8.0, 0.4)
    ratio_trunc = ec / er
    ratio_gold = gold_c / gold_r
    assert abs(ratio_gold - ratio_scaling) <= 6e-4 * ratio_gold
    assert abs(ratio_gold - ratio_trunc) >= 2e-2 * ratio_gold
    eps = gold_r / lapl_norm(a, b)
    assert 3.6e-5 <= eps <= 3.8e-5
    assert er <= 3.0e-3 and abs(er - gold_r) <= 3.0e-3


def test_reference_kernel_matches_restatement_when_built():
    from oracle import oracle as O
    if O.ref_operate() is None:
        pytest.skip("reference kernel not built here")
    from hpsi.stencil import laplacian_weights, star_points
    m, v, proj, psi = small_sphere_system(nst=4)
    w = laplacian_weights(m.spacing)
    a = O.Hamiltonian(m, w, star_points(), v=v, use_ref=True).apply(psi)
    b = O.Hamiltonian(m, w, star_points(), v=v, use_ref=False).apply(psi)
    assert rel_maxnorm_per_state(b, a) <= 1e-15


def test_mesh_sizes_of_benchmark_configs():
    from hpsi.mesh import index_box_mesh, sphere_mesh
    m0 = index_box_mesh((64, 64, 64), 0.25)
    assert (m0.np, m0.np_part) == (262144, 360448)
    m = sphere_mesh(8.0, 0.4)
    assert (m.np, m.np_part) == (33401, 52297)


def test_nl_operator_runs_reproduce_neighbours():
    from oracle import oracle as O
    from hpsi.mesh import sphere_mesh
    from hpsi.stencil import star_points
    m = sphere_mesh(2.4, 0.3)
    pts = star_points()
    nbr = O.neighbour_table(m, pts)
    op = O.Operator(m, pts)
    ri = op.ri.reshape(op.nri, op.W)
    for i in range(m.np):
        assert np.array_equal(ri[op.rimap[i]] + i, nbr[i])
    assert op.rimap_inv[0] == 0 and op.rimap_inv[-1] == m.np


def _dense_h(H, n):
    cols = []
    for i in range(n):
        e = np.zeros((H.mesh.np_part, 1), dtype=np.complex128)
        e[i, 0] = 1.0
        cols.append(H.apply(e)[:, 0])
    return np.stack(cols, axis=1)


def test_oracle_hamiltonian_hermitian_and_taylor_polynomial():
    """H (oracle, zero BC) is Hermitian on the inner points and the Taylor
    step equals the dense polynomial sum_k (-i dt H)^k / k! psi."""
    from oracle import oracle as O
    from hpsi import fixtures
    from hpsi.mesh import index_box_mesh
    from hpsi.stencil import laplacian_weights, star_points
    rng = np.random.default_rng(5)
    m = index_box_mesh((5, 4, 4), 0.3)
    v = fixtures.soft_coulomb(m, rng)
    proj = fixtures.kb_projectors(m, 1, rng, radius=0.5, min_dist=0.1, place_radius=0.1)
    P = O.Projectors(proj.maps, proj.mats, proj.scals)
    H = O.Hamiltonian(m, laplacian_weights(m.spacing), star_points(), v=v, projectors=P)
    Hd = _dense_h(H, m.np)
    # KB projector with the same P on both sides is symmetric; the stencil too
    assert np.max(np.abs(Hd - Hd.conj().T)) <= 1e-10 * np.max(np.abs(Hd))
    psi = np.zeros((m.np_part, 2), dtype=np.complex128)
    psi[: m.np] = rng.standard_normal((m.np, 2)) + 1j * rng.standard_normal((m.np, 2))
    dt = 0.01
    got = H.taylor(psi, dt, order=4)
    ref = psi[: m.np].copy()
    term = psi[: m.np].copy()
    for k in range(1, 5):
        term = (-1j * dt / k) * (Hd @ term)
        ref = ref + term
    assert rel_maxnorm_per_state(got, ref) <= 1e-13


def test_oracle_projector_matches_dense_formula():
    from oracle import oracle as O
    from hpsi.stencil import laplacian_weights, star_points
    m, v, proj, psi = small_sphere_system(nst=3)
    P = O.Projectors(proj.maps, proj.mats, proj.scals)
    w0 = np.zeros(25)
    H = O.Hamiltonian(m, w0, star_points(), v=None, projectors=P)
    got = H.apply(psi)
    ref = np.zeros_like(got)
    for mp, mat, sc in zip(proj.maps, proj.mats, proj.scals):
        pr = sc[:, None] * (mat.T @ psi[mp])
        ref[mp] += mat @ pr
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_density_restatement_matches_reference_loop():
    """oracle.density_accumulate against an explicit point/state double loop in
    the order of the reference's packed branch (density.F90:337-357)."""
    import numpy as np
    from hpsi.mesh import index_box_mesh
    from oracle import oracle as O
    m = index_box_mesh((5, 4, 3), 0.5)
    rng = np.random.default_rng(5)
    psi = rng.standard_normal((m.np_part, 3)) + 1j * rng.standard_normal((m.np_part, 3))
    w = rng.uniform(0, 2, 3)
    ref = np.zeros(m.np)
    for ip in range(m.np):
        for ist in range(3):
            ref[ip] += w[ist] * (np.conj(psi[ip, ist]) * psi[ip, ist]).real
    got = O.density_accumulate(m, psi, w)
    assert np.max(np.abs(got - ref)) <= 1e-14 * np.max(ref)


def test_lanczos_restatement_matches_dense_exponential():
    """The Lanczos restatement converges to exp(-i dt H) psi computed from the
    eigendecomposition of the dense oracle H (Hermitian on the inner points)."""
    from oracle import oracle as O
    from hpsi import fixtures
    from hpsi.mesh import index_box_mesh
    from hpsi.stencil import laplacian_weights, star_points
    rng = np.random.default_rng(7)
    m = index_box_mesh((5, 4, 4), 0.3)
    v = fixtures.soft_coulomb(m, rng)
    proj = fixtures.kb_projectors(m, 1, rng, radius=0.5, min_dist=0.1, place_radius=0.1)
    P = O.Projectors(proj.maps, proj.mats, proj.scals)
    H = O.Hamiltonian(m, laplacian_weights(m.spacing), star_points(), v=v, projectors=P)
    Hd = _dense_h(H, m.np)[: m.np]
    Hd = 0.5 * (Hd + Hd.conj().T)
    lam, Q = np.linalg.eigh(Hd)
    psi = np.zeros((m.np_part, 3), dtype=np.complex128)
    psi[: m.np] = rng.standard_normal((m.np, 3)) + 1j * rng.standard_normal((m.np, 3))
    for dt in (0.01, 0.2):
        ref = (Q * np.exp(-1j * dt * lam)[None, :]) @ (Q.conj().T @ psi[: m.np])
        got, mdim, res = O.lanczos(H, psi, dt, max_order=60, tol=1e-11)
        assert res < 1e-11 and mdim > 3
        assert rel_maxnorm_per_state(got, ref) <= 1e-9


def test_kb_with_projector_phases_is_hermitian():
    """The oracle's KB term with projector phases (k != 0) is a Hermitian
    operator, <a|K b> = <K a|b>, and unit phases give the plain term."""
    from helpers import small_sphere_system
    from oracle import oracle as O
    m, v, proj, psi = small_sphere_system(seed=67, nst=2, natoms=3)
    rng = np.random.default_rng(68)
    ph = [np.exp(1j * rng.uniform(0, 2 * np.pi, len(mp))) for mp in proj.maps]

    def K(x, phases):
        p = O.kb_bra(proj.maps, proj.mats, proj.scals, x, phases)
        return O.kb_ket(proj.maps, proj.mats, p, np.zeros((m.np, x.shape[1]), complex), phases)

    a, b = psi[: m.np, :1], psi[: m.np, 1:2]
    lhs = np.vdot(a, K(b, ph))
    rhs = np.vdot(K(a, ph), b)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    ones = [np.ones(len(mp)) for mp in proj.maps]
    x = psi[: m.np]
    assert np.allclose(K(x, ones), K(x, None), rtol=0, atol=1e-13 * np.abs(K(x, None)).max())
    assert np.abs(K(x, ph) - K(x, None)).max() > 1e-3 * np.abs(K(x, None)).max()


REF_GPU_GOLDEN = os.path.join(HERE, "golden", "ref_gpu_kernels.npz")


def _ref_gpu_golden():
    if not os.path.exists(REF_GPU_GOLDEN):
        pytest.skip("reference GPU kernel golden file not generated")
    g = np.load(REF_GPU_GOLDEN)
    from hpsi.fixtures import ProjectorSet
    from hpsi.mesh import Mesh
    m = Mesh(lxyz=g["lxyz"], np=int(g["np"]), spacing=g["spacing"])
    npts, nprj = g["npoints"], g["nprojs"]
    maps, mats, scals = [], [], []
    o = om = os_ = 0
    for a, b in zip(npts, nprj):
        maps.append(g["maps"][o: o + a])
        mats.append(g["mats"][om: om + a * b].reshape(a, b))
        scals.append(g["scals"][os_: os_ + b])
        o, om, os_ = o + a, om + a * b, os_ + b
    return g, m, ProjectorSet(maps, mats, scals, None)


def test_restated_kernels_match_reference_gpu_kernels():
    """The oracle's restatements of the stencil (times -1/2), vpsi, the KB bra
    and ket and the axpy against the reference's own GPU kernels
    (share/opencl operate.cl operate_map, vpsi.cl vpsi, projector.cl
    dprojector_bra/dprojector_ket, axpy.cl daxpy), built from source for
    sm_100a and run on a B200 (tests/golden/make_ref_gpu_golden.py)."""
    from oracle import oracle as O
    from hpsi.stencil import star_points
    g, m, proj = _ref_gpu_golden()
    psi = g["psi"]
    w = g["weights"]
    nst = psi.shape[1]
    kin = O.Hamiltonian(m, w, star_points(), v=None, use_ref=False).apply(psi)
    assert rel_maxnorm_per_state(kin[:, :4], g["kinetic"][:, :4]) <= 1e-13
    vpsi = g["v"][:, None] * psi[: m.np]
    assert np.max(np.abs(vpsi - g["vpsi"])) <= 1e-14 * np.max(np.abs(vpsi))
    pr = O.kb_bra(proj.maps, proj.mats, proj.scals, psi)
    assert np.max(np.abs(pr - g["projections"])) <= 1e-13 * np.max(np.abs(pr))
    ket = O.kb_ket(proj.maps, proj.mats, g["projections"], np.zeros((m.np, nst), complex))
    assert np.max(np.abs(ket - g["ket"])) <= 1e-13 * np.max(np.abs(ket))
    P = O.Projectors(proj.maps, proj.mats, proj.scals)
    h = O.Hamiltonian(m, w, star_points(), v=g["v"], projectors=P, use_ref=False).apply(psi[:, :4])
    assert rel_maxnorm_per_state(h, g["hpsi"][:, :4]) <= 1e-13
    ax = g["axpy_in"] + float(g["axpy_a"]) * psi[: m.np]
    assert np.max(np.abs(ax - g["axpy_out"])) <= 1e-15 * np.max(np.abs(ax))
