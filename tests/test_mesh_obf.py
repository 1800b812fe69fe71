"""The mesh order on disk (the reference's restart file indices.obf): cubic
spatial indices, the io_binary header, and parity with the reference's own
binary I/O (a golden file it wrote, and, where oracle/_ref holds the
reference's io_binary.c built from source, its reader on our file)."""
import ctypes as C
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "indices_sphere_r1.5_h0.3.obf")
REF_IO = os.path.join(ROOT, "oracle", "_ref", "libref_io_binary.so")


def _meshes():
    from hpsi.mesh import index_box_mesh, parallelepiped_mesh, sphere_mesh
    return [sphere_mesh(1.5, 0.3), sphere_mesh(3.0, 0.25), parallelepiped_mesh([1.0, 1.5, 0.75], 0.25),
            index_box_mesh((6, 5, 4), 0.3)]


@pytest.mark.parametrize("k", range(4))
def test_cubic_index_round_trip(k):
    from hpsi.mesh import cubic_extent, cubic_index, cubic_point
    m = _meshes()[k]
    e = cubic_extent(m)
    idx = cubic_index(m.lxyz, e)
    assert np.unique(idx).shape[0] == m.np_part
    assert idx.min() >= 0 and idx.max() < np.prod(2 * e + 1)
    assert np.array_equal(cubic_point(idx, e), m.lxyz)
    with pytest.raises(ValueError):
        cubic_index(m.lxyz, e - 1)


def test_writer_is_byte_identical_to_the_reference_file(tmp_path):
    from hpsi.mesh import sphere_mesh, write_indices_obf
    p = tmp_path / "indices.obf"
    write_indices_obf(p, sphere_mesh(1.5, 0.3))
    assert p.read_bytes() == open(GOLDEN, "rb").read()


def test_reader_recovers_the_mesh_from_the_reference_file():
    from hpsi.mesh import mesh_from_indices_obf, read_indices_obf, sphere_mesh
    m = sphere_mesh(1.5, 0.3)
    assert read_indices_obf(GOLDEN).shape == (m.np_part,)
    m2 = mesh_from_indices_obf(GOLDEN, m.np, m.spacing, [9, 9, 9])
    assert m2.np == m.np and np.array_equal(m2.lxyz, m.lxyz)


def test_reader_converts_big_endian_files(tmp_path):
    from hpsi.mesh import read_indices_obf
    from hpsi.obf import HEADER as _OBF_HEADER
    raw = open(GOLDEN, "rb").read()
    h = np.frombuffer(raw[:64], dtype=_OBF_HEADER).astype(_OBF_HEADER.newbyteorder(">"))
    n = int(h["np"][0])
    vals = np.frombuffer(raw[64:], dtype="<i8").astype(">i8")
    p = tmp_path / "be.obf"
    p.write_bytes(h.tobytes() + vals.tobytes())
    assert np.array_equal(read_indices_obf(p), read_indices_obf(GOLDEN))
    assert read_indices_obf(p).shape == (n,)


def test_reader_rejects_bad_files(tmp_path):
    from hpsi.mesh import read_indices_obf
    raw = bytearray(open(GOLDEN, "rb").read())
    cases = {"short": bytes(raw[:40]), "text": b"pulpX" + bytes(raw[5:]),
             "truncated": bytes(raw[:64 + 8 * 10])}
    bad_type = bytearray(raw)
    bad_type[40:44] = (3).to_bytes(4, "little")   # TYPE_DOUBLE_COMPLEX payload
    cases["type"] = bytes(bad_type)
    for name, data in cases.items():
        p = tmp_path / f"{name}.obf"
        p.write_bytes(data)
        with pytest.raises(ValueError):
            read_indices_obf(p)


@pytest.mark.skipif(not os.path.exists(REF_IO), reason="reference io_binary.c not built (make -C oracle ref)")
def test_reference_reader_reads_our_file(tmp_path):
    from hpsi.mesh import IO_TYPE_INT_64, cubic_extent, cubic_index, sphere_mesh, write_indices_obf
    lib = C.CDLL(REF_IO)
    m = sphere_mesh(3.0, 0.25)
    p = tmp_path / "indices.obf"
    write_indices_obf(p, m)
    fname = C.c_char_p(os.fsencode(str(p)))
    n, typ, size, ierr, iio = C.c_int64(0), C.c_int(0), C.c_int64(0), C.c_int(0), C.c_int(0)
    lib.get_info_binary(C.byref(n), C.byref(typ), C.byref(size), C.byref(ierr), C.byref(iio), fname)
    assert ierr.value == 0 and n.value == m.np_part and typ.value == IO_TYPE_INT_64
    out = np.zeros(m.np_part, dtype=np.int64)
    off, otyp = C.c_int64(0), C.c_int(IO_TYPE_INT_64)
    lib.read_binary(C.byref(n), C.byref(off), out.ctypes.data_as(C.c_void_p), C.byref(otyp), C.byref(ierr),
                    C.byref(iio), fname)
    assert ierr.value == 0
    assert np.array_equal(out, cubic_index(m.lxyz, cubic_extent(m)))


GOLDEN_HILBERT = os.path.join(ROOT, "tests", "golden", "indices_hilbert_sphere_r1.5_h0.3.obf")
REF_HILBERT = os.path.join(ROOT, "oracle", "_ref", "libref_hilbert.so")


@pytest.mark.parametrize("k", range(4))
def test_hilbert_index_round_trip(k):
    from hpsi.mesh import cubic_extent, hilbert_bits, hilbert_index, hilbert_point
    m = _meshes()[k]
    e = cubic_extent(m)
    idx = hilbert_index(m.lxyz, e)
    assert np.unique(idx).shape[0] == m.np_part
    assert idx.min() >= 0 and idx.max() < 1 << (3 * hilbert_bits(e))
    assert np.array_equal(hilbert_point(idx, e), m.lxyz)


def test_hilbert_curve_is_continuous():
    """Consecutive Hilbert indices are neighbouring grid points."""
    from hpsi.mesh import hilbert_point
    e = np.array([3, 3, 3])  # grid 7^3 inside the 8^3 curve
    pts = hilbert_point(np.arange(8 ** 3), e).astype(np.int64)
    assert np.all(np.abs(np.diff(pts, axis=0)).sum(axis=1) == 1)


def test_hilbert_file_matches_the_reference_golden(tmp_path):
    from hpsi.mesh import mesh_from_indices_obf, sphere_mesh, write_indices_obf
    m = sphere_mesh(1.5, 0.3)
    p = tmp_path / "h.obf"
    write_indices_obf(p, m, index_type="hilbert")
    assert p.read_bytes() == open(GOLDEN_HILBERT, "rb").read()
    m2 = mesh_from_indices_obf(GOLDEN_HILBERT, m.np, m.spacing, [9, 9, 9], index_type="hilbert")
    assert np.array_equal(m2.lxyz, m.lxyz)


@pytest.mark.skipif(not os.path.exists(REF_HILBERT), reason="reference hilbert.c not built (make -C oracle ref)")
def test_hilbert_matches_the_reference_kernel():
    from hpsi.mesh import hilbert_bits, hilbert_index, hilbert_point
    lib = C.CDLL(REF_HILBERT)
    rng = np.random.default_rng(5)
    for e in ([9, 9, 9], [12, 7, 20], [30, 30, 30]):
        e = np.asarray(e)
        pts = rng.integers(-e, e + 1, size=(400, 3))
        ours = hilbert_index(pts, e)
        dim, nb, idx = C.c_int(3), C.c_int(hilbert_bits(e)), C.c_longlong(0)
        off = (2 * e + 1) // 2
        for p, h in zip(pts + off, ours):
            pt = (C.c_int * 3)(*[int(v) for v in p])
            lib.hilbert_point_to_index_(C.byref(dim), C.byref(nb), C.byref(idx), pt)
            assert idx.value == h
            back = (C.c_int * 3)()
            lib.hilbert_index_to_point_(C.byref(dim), C.byref(nb), C.byref(C.c_longlong(int(h))), back)
            assert list(back) == [int(v) for v in p]
        assert np.array_equal(hilbert_point(ours, e), pts)


@pytest.mark.parametrize("dt", ["f4", "f8", "c8", "c16", "i4", "i8"])
def test_obf_round_trip_every_type(tmp_path, dt):
    from hpsi.obf import read_obf, write_obf
    rng = np.random.default_rng(3)
    v = (rng.standard_normal(37) * 100).astype(dt) if dt[0] in "fi" else \
        (rng.standard_normal(37) + 1j * rng.standard_normal(37)).astype(dt)
    p = tmp_path / "v.obf"
    write_obf(p, v)
    got = read_obf(p)
    assert got.dtype == np.dtype(dt) and np.array_equal(got, v)
    with pytest.raises(ValueError):
        write_obf(tmp_path / "e.obf", v[:0])


@pytest.mark.skipif(not os.path.exists(REF_IO), reason="reference io_binary.c not built (make -C oracle ref)")
def test_state_files_both_ways_with_the_reference(tmp_path):
    """Complex and real mesh functions: files the reference's write_binary
    makes load into a batch (real ones widened as its read_binary converts
    them), and the reference's read_binary reads write_obf's files."""
    from hpsi.mesh import sphere_mesh
    from hpsi.obf import TYPE_DOUBLE, TYPE_DOUBLE_COMPLEX, load_states_obf, write_obf
    lib = C.CDLL(REF_IO)
    m = sphere_mesh(1.5, 0.3)
    rng = np.random.default_rng(7)
    states = [rng.standard_normal(m.np) + 1j * rng.standard_normal(m.np) for _ in range(2)]
    states.append(rng.standard_normal(m.np))          # a real state (gs restart of a real run)
    paths = []
    for i, s in enumerate(states):
        p = tmp_path / f"{i + 1:010d}.obf"
        v = np.ascontiguousarray(s)
        n = C.c_int64(m.np)
        typ = C.c_int(TYPE_DOUBLE_COMPLEX if np.iscomplexobj(v) else TYPE_DOUBLE)
        ierr, iio, nhd, flpe = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
        lib.write_binary(C.byref(n), v.ctypes.data_as(C.c_void_p), C.byref(typ), C.byref(ierr), C.byref(iio),
                         C.byref(nhd), C.byref(flpe), C.c_char_p(os.fsencode(str(p))))
        assert ierr.value == 0
        paths.append(p)
    b = load_states_obf(paths, m, ld=4)
    assert b.shape == (m.np_part, 4) and not b[m.np:].any() and not b[:, 3].any()
    for i, s in enumerate(states):
        assert np.array_equal(b[: m.np, i], s.astype(np.complex128))
    # the reference's reader, asked for complex output, on the real file and on write_obf's file
    for src in (paths[2], tmp_path / "ours.obf"):
        if src == tmp_path / "ours.obf":
            write_obf(src, states[0])
        out = np.zeros(m.np, dtype=np.complex128)
        n, off, otyp = C.c_int64(m.np), C.c_int64(0), C.c_int(TYPE_DOUBLE_COMPLEX)
        ierr, iio = C.c_int(0), C.c_int(0)
        lib.read_binary(C.byref(n), C.byref(off), out.ctypes.data_as(C.c_void_p), C.byref(otyp), C.byref(ierr),
                        C.byref(iio), C.c_char_p(os.fsencode(str(src))))
        want = states[2].astype(np.complex128) if src == paths[2] else states[0]
        assert np.array_equal(out, want), ierr.value


def test_load_states_rejects_wrong_sizes(tmp_path):
    from hpsi.mesh import sphere_mesh
    from hpsi.obf import load_states_obf, write_obf
    m = sphere_mesh(1.5, 0.3)
    write_obf(tmp_path / "a.obf", np.zeros(m.np + 1, dtype=np.complex128))
    write_obf(tmp_path / "i.obf", np.zeros(m.np, dtype=np.int64))
    for name in ("a.obf", "i.obf"):
        with pytest.raises(ValueError):
            load_states_obf([tmp_path / name], m)
    with pytest.raises(ValueError):
        load_states_obf([tmp_path / "a.obf"] * 2, m, ld=1)


def test_save_and_load_states_round_trip(tmp_path):
    import torch
    from hpsi.mesh import sphere_mesh
    from hpsi.obf import load_states_obf, read_obf, save_states_obf
    m = sphere_mesh(1.5, 0.3)
    rng = np.random.default_rng(11)
    b = np.zeros((m.np_part, 4), dtype=np.complex64)
    b[: m.np, :3] = rng.standard_normal((m.np, 3)) + 1j * rng.standard_normal((m.np, 3))
    paths = [tmp_path / f"{i + 1:010d}.obf" for i in range(3)]
    save_states_obf(torch.from_numpy(b), m, paths)
    assert read_obf(paths[0]).dtype == np.complex64
    got = load_states_obf(paths, m, ld=4, dtype=np.complex64)
    assert np.array_equal(got, b)
    with pytest.raises(ValueError):
        save_states_obf(b[:, :2], m, paths)


REF_CK = os.path.join(ROOT, "oracle", "_ref", "libref_checksum.so")


@pytest.mark.parametrize("index_type", ["cubic", "hilbert"])
def test_mesh_from_restart_directory(tmp_path, index_type):
    """A restart directory as the reference leaves it (the "grid"
    fingerprint and indices.obf) gives back the mesh; a wrong checksum is
    refused."""
    from hpsi.mesh import (mesh_from_restart, read_grid_fingerprint, sphere_mesh, write_grid_fingerprint,
                           write_indices_obf)
    m = sphere_mesh(2.0, 0.25)
    write_indices_obf(tmp_path / "indices.obf", m, index_type=index_type)
    write_grid_fingerprint(tmp_path / "grid", m, index_type=index_type)
    lines = (tmp_path / "grid").read_text().splitlines()
    assert len(lines) == 13 and all(len(ln) == 41 for ln in lines)
    assert lines[7].startswith("offset( 1)=") and lines[10].startswith("    nn( 1)=")
    fp = read_grid_fingerprint(tmp_path / "grid")
    assert fp["np"] == m.np and fp["np_part"] == m.np_part and fp["type"] == (1 if index_type == "cubic" else 2)
    m2 = mesh_from_restart(tmp_path, m.spacing)
    assert m2.np == m.np and np.array_equal(m2.lxyz, m.lxyz)
    bad = lines[:3] + [f"{'checksum=':<20s}{fp['checksum'] + 1:21d}"] + lines[4:]
    (tmp_path / "grid").write_text("\n".join(bad) + "\n")
    with pytest.raises(ValueError):
        mesh_from_restart(tmp_path, m.spacing)


@pytest.mark.skipif(not os.path.exists(REF_CK), reason="reference checksum.c not built (make -C oracle ref)")
def test_index_checksum_matches_the_reference():
    from hpsi.mesh import index_checksum
    lib = C.CDLL(REF_CK)
    rng = np.random.default_rng(13)
    for n in (1, 10, 5000):
        for hi in (100, 1 << 40, (1 << 62)):   # the last case wraps around 2^64
            v = rng.integers(0, hi, size=n, dtype=np.int64)
            alg, nn, s = C.c_int(1), C.c_int64(n), C.c_int64(0)
            lib.checksum_calculate_(C.byref(alg), C.byref(nn), v.ctypes.data_as(C.c_void_p), C.byref(s))
            assert index_checksum(v) == s.value
