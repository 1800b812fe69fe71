"""KB projector phases (k != 0): the bra gathers psi(map) * phase, the ket
adds its contribution times conj(phase)
(src/hamiltonian/hamiltonian_elec_base_inc.F90:680-701, 934-1025).  The KB
term of the device H psi (all terms minus kinetic + local) is compared with
a numpy restatement of those two steps."""
import numpy as np
import pytest

from helpers import small_sphere_system

pytestmark = pytest.mark.gpu


def _kb_with_phases(proj, phases, psi, np_inner):
    h = np.zeros((np_inner, psi.shape[1]), dtype=np.complex128)
    for mp, mt, sc, ph in zip(proj.maps, proj.mats, proj.scals, phases):
        lpsi = psi[mp] * ph[:, None]
        pr = np.asarray(sc)[:, None] * (np.asarray(mt).T @ lpsi)
        np.add.at(h, mp, (np.asarray(mt) @ pr) * np.conj(ph)[:, None])
    return h


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_kb_term_with_projector_phases(cuda, dtype):
    import torch
    from hpsi import lib
    from hpsi.stencil import laplacian_weights, star_points
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    nst = 8
    m, v, proj, psi = small_sphere_system(seed=61, nst=nst, radius=4.0, natoms=3)
    rng = np.random.default_rng(62)
    phases = [np.exp(1j * rng.uniform(0, 2 * np.pi, len(mp))) for mp in proj.maps]
    H = lib.Hamiltonian(lib.DeviceMesh(m), laplacian_weights(m.spacing), star_points(), v=v, projectors=proj)
    H.set_projector_phases(phases)
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
