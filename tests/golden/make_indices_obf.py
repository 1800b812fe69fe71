"""Generate the indices.obf golden file with the reference's own binary I/O.

Run in a container where the reference sources are present:

    make -C oracle ref REF=<reference source tree> && python tests/golden/make_indices_obf.py

It loads oracle/_ref/libref_io_binary.so and oracle/_ref/libref_hilbert.so
(the reference's src/basic/io_binary.c and src/grid/hilbert.c built from
source) and writes, through its ``write_binary`` (header + payload, as
index_dump does, src/grid/index.F90:176-200), the spatial indices of the
points of a small sphere mesh (R = 1.5, h = 0.3, order 4) in mesh order:
the cubic indices (idx_cubic), and the Hilbert indices (idx_hilbert) that
the reference's ``hilbert_point_to_index`` gives for the offset points.  The tests
compare this library's writer and reader against the file on machines
without the reference.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "octopus-debian-package_b200"))

from hpsi.mesh import IO_TYPE_INT_64, cubic_extent, cubic_index, sphere_mesh  # noqa: E402

OUT = os.path.join(HERE, "indices_sphere_r1.5_h0.3.obf")
OUT_HILBERT = os.path.join(HERE, "indices_hilbert_sphere_r1.5_h0.3.obf")


def reference_hilbert(lxyz, extent):
    from hpsi.mesh import hilbert_bits
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_hilbert.so"))
    e = np.asarray(extent, dtype=np.int64)
    off = (2 * e + 1) // 2
    dim, nb, idx = C.c_int(3), C.c_int(hilbert_bits(e)), C.c_longlong(0)
    out = np.empty(len(lxyz), dtype=np.int64)
    for i, p in enumerate(np.asarray(lxyz, dtype=np.int64) + off):
        pt = (C.c_int * 3)(*[int(v) for v in p])
        lib.hilbert_point_to_index_(C.byref(dim), C.byref(nb), C.byref(idx), pt)
        out[i] = idx.value
    return out


def reference_write(path, values):
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_io_binary.so"))
    v = np.ascontiguousarray(values, dtype=np.int64)
    n = C.c_int64(v.shape[0])
    typ, ierr, iio, nhd, flpe = C.c_int(IO_TYPE_INT_64), C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
    lib.write_binary(C.byref(n), v.ctypes.data_as(C.c_void_p), C.byref(typ), C.byref(ierr), C.byref(iio),
                     C.byref(nhd), C.byref(flpe), C.c_char_p(os.fsencode(path)))
    if ierr.value != 0:
        raise RuntimeError(f"write_binary failed: {ierr.value}")


def main():
    m = sphere_mesh(1.5, 0.3)
    reference_write(OUT, cubic_index(m.lxyz, cubic_extent(m)))
    reference_write(OUT_HILBERT, reference_hilbert(m.lxyz, cubic_extent(m)))
    print(OUT, m.np, m.np_part, cubic_extent(m))


if __name__ == "__main__":
    main()
