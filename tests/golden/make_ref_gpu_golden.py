"""Golden vectors from the reference's own GPU kernels (share/opencl, compiled
for sm_100a by oracle/refgpu_build.py and launched by oracle/refgpu.py as the
reference launches them).  Needs a GPU and the CUBINs in oracle/_ref:

    python oracle/refgpu_build.py <reference source tree>     # here
    python tests/golden/make_ref_gpu_golden.py <out.npz>       # on a GPU

Records, for a small seeded sphere system (R = 3.6 bohr, h = 0.3, 3 KB atoms,
4 complex128 states in an 8-wide packed batch), the output of each kernel on
its own -- operate_map (kinetic, weights times -1/2), vpsi, dprojector_bra
(projections), dprojector_ket (ket added to zero), daxpy -- and of the whole
H.psi in the reference's order.  tests/test_oracle.py compares the CPU
restatements with this file.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "octopus-debian-package_b200"))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def main(out_path):
    import torch
    from helpers import small_sphere_system
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import refgpu
    dev = torch.device("cuda", 0)
    m, v, proj, psi = small_sphere_system(seed=5, nst=4, radius=3.6, spacing=0.3, natoms=3)
    ld = 8
    x = np.zeros((m.np_part, ld), dtype=np.complex128)
    x[:, :4] = psi
    w = laplacian_weights(m.spacing)
    R = refgpu.RefHamiltonian(m, w, star_points(), v, proj, dev)
    xt = torch.from_numpy(x).to(dev)
    kin = torch.zeros((m.np, ld), dtype=torch.complex128, device=dev)
    R.kinetic(xt, kin)
    loc = torch.zeros_like(kin)
    R.local(xt, loc)
    pr = R.projection_buffer(xt)
    R.bra(xt, pr)
    ket = torch.zeros_like(kin)
    R.ket(pr, ket)
    h = torch.zeros_like(kin)
    R.apply(xt, h)
    rng = np.random.default_rng(6)
    ya = rng.standard_normal((m.np, ld)) + 1j * rng.standard_normal((m.np, ld))
    yt = torch.from_numpy(ya).to(dev)
    R.axpy(-0.37, xt, yt)
    torch.cuda.synchronize()
    # the 4 states in use (columns 4..7 of the packed batch are padding)
    c4 = lambda a: np.ascontiguousarray(a[:, :4])  # noqa: E731
    np.savez_compressed(
        out_path, lxyz=m.lxyz, np=np.int64(m.np), spacing=m.spacing, weights=w, v=v, psi=c4(x),
        maps=np.concatenate(proj.maps), npoints=np.array([len(a) for a in proj.maps]),
        mats=np.concatenate([np.asarray(a, dtype=np.float64).ravel() for a in proj.mats]),
        nprojs=np.array([a.shape[1] for a in proj.mats]), scals=np.concatenate(proj.scals),
        kinetic=c4(kin.cpu().numpy()), vpsi=c4(loc.cpu().numpy()),
        projections=c4(pr.cpu().numpy().view(np.complex128)), ket=c4(ket.cpu().numpy()),
        hpsi=c4(h.cpu().numpy()), axpy_in=c4(ya), axpy_a=np.float64(-0.37), axpy_out=c4(yt.cpu().numpy()))
    print("wrote", out_path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_gpu_kernels.npz"))
