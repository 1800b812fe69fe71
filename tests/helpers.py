"""Shared helpers of the test-suite (numerics tolerances, small systems)."""
import numpy as np


def rel_maxnorm_per_state(got, ref):
    """max over states of max_ip |got - ref| / max_ip |ref| (the parity metric)."""
    got = np.asarray(got)
    ref = np.asarray(ref)
    num = np.max(np.abs(got - ref), axis=0)
    den = np.max(np.abs(ref), axis=0)
    den = np.where(den == 0, 1.0, den)
    return float(np.max(num / den))


def small_sphere_system(seed=3, nst=6, radius=3.6, spacing=0.3, natoms=3):
    from hpsi import fixtures
    from hpsi.mesh import sphere_mesh
    rng = np.random.default_rng(seed)
    m = sphere_mesh(radius, spacing)
    v = fixtures.soft_coulomb(m, rng)
    proj = fixtures.kb_projectors(m, natoms, rng, radius=1.2, min_dist=1.0, place_radius=1.5)
    psi = fixtures.random_states(m, nst, rng)
    return m, v, proj, psi
