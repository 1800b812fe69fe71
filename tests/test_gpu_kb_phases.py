"""KB projector phases (k != 0): the bra gathers psi(map) * phase, the ket
adds its contribution times conj(phase)
(src/hamiltonian/hamiltonian_elec_base_inc.F90:680-701, 934-1025).  The KB
term of the device H psi (all terms minus kinetic + local), a Taylor step and
the split bra/ket entry points are compared with a numpy restatement of those
two steps (plus the oracle's kinetic + local H for the Taylor step).

Batch widths 8 and 40: with 40 states (80 real lanes) the bra's lane-pair
exchange spans several thread-block rows; the phases are passed both packed
and in the reference's padded projector_phases(:, 1, :, ik) layout."""
import numpy as np
import pytest

from helpers import rel_maxnorm_per_state, small_sphere_system

pytestmark = pytest.mark.gpu


def _kb_with_phases(proj, phases, psi, np_inner):
    h = np.zeros((np_inner, psi.shape[1]), dtype=np.complex128)
    for mp, mt, sc, ph in zip(proj.maps, proj.mats, proj.scals, phases):
        lpsi = psi[mp] * ph[:, None]
        pr = np.asarray(sc)[:, None] * (np.asarray(mt).T @ lpsi)
        np.add.at(h, mp, (np.asarray(mt) @ pr) * np.conj(ph)[:, None])
    return h


def _system(nst, seed=61):
    m, v, proj, psi = small_sphere_system(seed=seed, nst=nst, radius=4.0, natoms=3)
    rng = np.random.default_rng(seed + 1)
    phases = [np.exp(1j * rng.uniform(0, 2 * np.pi, len(mp))) for mp in proj.maps]
    return m, v, proj, psi, phases


def _padded(phases, ld_points):
    out = np.zeros((len(phases), ld_points), dtype=np.complex128)
    for i, ph in enumerate(phases):
        out[i, : len(ph)] = ph
        out[i, len(ph):] = np.nan  # padding is never read
    return out


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("nst", [8, 40])
@pytest.mark.parametrize("layout", ["packed", "padded"])
def test_kb_term_with_projector_phases(cuda, dtype, nst, layout):
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    m, v, proj, psi, phases = _system(nst)
    H = lib.Hamiltonian(lib.DeviceMesh(m), laplacian_weights(m.spacing), star_points(), v=v, projectors=proj)
    if layout == "packed":
        H.set_projector_phases(phases)
    else:
        ldp = max(len(p) for p in phases) + 3
        H.set_projector_phases(_padded(phases, ldp), ld_points=ldp)
    x = torch.from_numpy(psi).to(cuda).to(tdt)
    full = torch.zeros((m.np, nst), dtype=tdt, device=cuda)
    loc = torch.zeros((m.np, nst), dtype=tdt, device=cuda)
    H.apply(x, full)
    H.apply(x, loc, terms=lib.TERM_KINETIC | lib.TERM_LOCAL_POTENTIAL)
    got = (full - loc).cpu().numpy().astype(np.complex128)
    ref = _kb_with_phases(proj, phases, psi, m.np)
    tol = 1e-12 if dtype == "c128" else 2e-5
    scale = np.max(np.abs(full.cpu().numpy()))
    assert np.max(np.abs(got - ref)) <= tol * scale
    # unit phases give the plain KB term; removing the phases restores it too
    H.set_projector_phases([np.ones(len(mp)) for mp in proj.maps])
    one = torch.zeros_like(full)
    H.apply(x, one)
    H.set_projector_phases(None)
    plain = torch.zeros_like(full)
    H.apply(x, plain)
    assert (one - plain).abs().max().item() <= tol * scale


def test_projector_phases_layout_errors(cuda):
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    m, v, proj, psi, phases = _system(8)
    H = lib.Hamiltonian(lib.DeviceMesh(m), laplacian_weights(m.spacing), star_points(), v=v, projectors=proj)
    with pytest.raises(ValueError):
        H.set_projector_phases(np.concatenate(phases)[:-1])  # one phase short
    ldp = max(len(p) for p in phases)
    with pytest.raises(ValueError):
        H.set_projector_phases(_padded(phases, ldp), ld_points=ldp - 1)
    # the C side rejects a stride below the largest sphere by itself
    import ctypes as C
    flat = np.ascontiguousarray(_padded(phases, ldp).ravel())
    st = lib.load().hpsi_hamiltonian_set_projector_phases(H.handle, flat.ctypes.data_as(C.POINTER(C.c_double)),
                                                          ldp - 1)
    assert st == 1


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_taylor_step_with_projector_phases(cuda, dtype):
    """psi <- sum_k (-i dt H)^k / k! psi with H = kinetic + local (oracle) +
    KB with phases (restatement), against the device Taylor step."""
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O
    nst = 40
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    m, v, proj, psi, phases = _system(nst, seed=71)
    w = laplacian_weights(m.spacing)
    H = lib.Hamiltonian(lib.DeviceMesh(m), w, star_points(), v=v, projectors=proj)
    H.set_projector_phases(phases)
    Hl = O.Hamiltonian(m, w, star_points(), v=v)

    def happ(x_inner):
        xp = np.zeros((m.np_part, nst), dtype=np.complex128)
        xp[: m.np] = x_inner
        return Hl.apply(xp) + _kb_with_phases(proj, phases, xp, m.np)

    dt = 0.01
    ref = psi[: m.np].copy()
    term = psi[: m.np].copy()
    for k in range(1, 5):
        term = (-1j * dt / k) * happ(term)
        ref = ref + term
    x = torch.from_numpy(psi).to(cuda).to(tdt)
    H.taylor_step(x, dt)
    got = x[: m.np].cpu().numpy().astype(np.complex128)
    tol = 1e-12 if dtype == "c128" else 2e-5
    assert rel_maxnorm_per_state(got, ref) <= tol


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_projector_bra_ket_with_phases(cuda, dtype):
    """hpsi_projector_bra / hpsi_projector_ket with phases set: projections and
    the ket's addition against the restatement (a = 1 and a complex factor)."""
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O
    nst = 40
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    m, v, proj, psi, phases = _system(nst, seed=81)
    H = lib.Hamiltonian(lib.DeviceMesh(m), laplacian_weights(m.spacing), star_points(), v=v, projectors=proj)
    H.set_projector_phases(phases)
    x = torch.from_numpy(psi).to(cuda).to(tdt)
    pr = torch.zeros((H.nprojections(), nst), dtype=tdt, device=cuda)
    H.projector_bra(x, pr)
    ref_pr = O.kb_bra(proj.maps, proj.mats, proj.scals, psi, phases)
    tol = 1e-12 if dtype == "c128" else 2e-5
    got_pr = pr.cpu().numpy().astype(np.complex128)
    assert np.max(np.abs(got_pr - ref_pr)) <= tol * np.max(np.abs(ref_pr))
    a = 0.3 - 0.7j
    base = np.asarray(psi[: m.np] * 0.5)
    out = torch.from_numpy(np.ascontiguousarray(base)).to(cuda).to(tdt)
    H.projector_ket(pr, out, a=a)
    ref = base + a * O.kb_ket(proj.maps, proj.mats, ref_pr, np.zeros((m.np, nst), complex), phases)
    assert rel_maxnorm_per_state(out.cpu().numpy().astype(np.complex128), ref) <= tol
