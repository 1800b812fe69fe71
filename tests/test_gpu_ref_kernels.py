"""The library against the reference's own GPU kernels on the same B200.

The reference's share/opencl kernels (operate_map, vpsi, dprojector_bra,
dprojector_ket), compiled from source for sm_100a by oracle/refgpu_build.py
and launched as the reference launches them (oracle/refgpu.py), give the
reference's GPU H.psi of the full headline system: sphere R = 12 bohr,
h = 0.2 (904,089 points), 32 KB atoms x 9 projectors, 128 complex128 states.
The library's H.psi of the same batch agrees per state to 1e-12 (relative
max-norm) over the whole batch."""
import numpy as np
import pytest

from helpers import rel_maxnorm_per_state

pytestmark = pytest.mark.gpu


def test_hpsi_matches_reference_gpu_kernels_full_size(cuda):
    import torch
    from oracle import refgpu
    if not refgpu.available():
        pytest.skip("reference kernels not built (oracle/refgpu_build.py)")
    from hpsi import fixtures, lib
    from hpsi.stencil import laplacian_weights, star_points
    s = fixtures.config1()
    m = s.mesh
    w = laplacian_weights(m.spacing)
    x = torch.from_numpy(s.psi).to(cuda)
    R = refgpu.RefHamiltonian(m, w, star_points(), s.v, s.proj, cuda)
    ref = torch.zeros((m.np, x.shape[1]), dtype=torch.complex128, device=cuda)
    R.apply(x, ref)
    H = lib.Hamiltonian(lib.DeviceMesh(m), w, star_points(), v=s.v, projectors=s.proj)
    y = torch.zeros_like(ref)
    H.apply(x, y)
    torch.cuda.synchronize()
    err = rel_maxnorm_per_state(y.cpu().numpy(), ref.cpu().numpy())
    assert err <= 1e-12, f"relative max-norm {err:.3e}"
