"""Generate golden vectors from the reference's own compiled stencil kernel.

Run in a container where the reference sources are present:

    make -C oracle ref REF=<reference source tree> && python tests/golden/make_golden.py

It compiles nothing itself; it loads oracle/_ref/libref_operate.so (the
reference's src/grid/operate.c built from source) and records, for small seeded
inputs, the output of `doperate_ri_vec_` with the solved order-4 weights times
-1/2 (the kinetic factor), plus the Laplacian error norm of the reference's
derivatives test (src/grid/derivatives_inc.F90:378-492) on its own mesh
(sphere R = 8, h = 0.4).  The tests compare the oracle restatement against
these files on machines without the reference.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "octopus-debian-package_b200"))
sys.path.insert(0, ROOT)

from hpsi.mesh import index_box_mesh, sphere_mesh  # noqa: E402
from hpsi.stencil import laplacian_weights, star_points  # noqa: E402
from oracle import oracle as O  # noqa: E402


def ref_stencil(mesh, w, x, ld):
    fn = O.ref_operate()
    if fn is None:
        raise SystemExit("oracle/_ref/libref_operate.so missing: run `make -C oracle ref REF=<reference source tree>` first")
    op = O.Operator(mesh, star_points())
    wre = np.ascontiguousarray(w * -0.5)
    fi = np.ascontiguousarray(x)
    fo = np.zeros((mesh.np, ld), dtype=np.complex128)
    ldf = int(np.log2(2 * ld))
    fn(C.byref(C.c_int(op.W)), O._p(wre), C.byref(C.c_int(op.nri)), O._p(op.ri, C.c_int), O._p(op.imin, C.c_int),
       O._p(op.imax, C.c_int), O._p(fi.view(np.float64)), C.byref(C.c_int(ldf)), O._p(fo.view(np.float64)))
    return fo


def main():
    rng = np.random.default_rng(2024)
    out = {}
    for name, m in (("sphere", sphere_mesh(2.4, 0.3)), ("box", index_box_mesh((7, 6, 5), 0.25))):
        ld = 4
        x = np.zeros((m.np_part, ld), dtype=np.complex128)
        x[:, :3] = rng.standard_normal((m.np_part, 3)) + 1j * rng.standard_normal((m.np_part, 3))
        w = laplacian_weights(m.spacing)
        out[f"{name}_lxyz"] = m.lxyz
        out[f"{name}_np"] = np.int64(m.np)
        out[f"{name}_spacing"] = m.spacing
        out[f"{name}_weights"] = w
        out[f"{name}_in"] = x
        out[f"{name}_out"] = ref_stencil(m, w, x, ld)
    m = sphere_mesh(8.0, 0.4)
    m.extra["bbox_l"] = 8.0
    w = laplacian_weights(0.4)
    out["deriv_real"] = np.float64(O.derivatives_test_error(m, w, star_points(), False, use_ref=True))
    out["deriv_complex"] = np.float64(O.derivatives_test_error(m, w, star_points(), True, use_ref=True))
    np.savez_compressed(os.path.join(HERE, "ref_operate.npz"), **out)
    print("wrote ref_operate.npz", {k: v.shape for k, v in out.items() if hasattr(v, "shape")})


if __name__ == "__main__":
    main()
