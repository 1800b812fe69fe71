"""Files in the reference's binary restart format (".obf", src/basic/io_binary.c).

A 64-byte header -- "pulpo", format version 0, the value one as uint32,
float, uint64 and double (the reader's endianness check), the element count
and a type code (src/basic/io_binary.c:112-150) -- followed by the values.
The reference writes mesh functions this way: the states of a restart
directory, one file per state over the np_global inner points in mesh order
(X(restart_write_mesh_function), src/grid/restart_inc.F90:21-97), and the
mesh order itself (indices.obf, src/grid/index.F90:176-200).

``read_obf`` / ``write_obf`` read and write any payload type;
``load_states_obf`` packs the state files of a restart directory into a
batch for the library (inner rows from the files, boundary rows zero), real
files widened to complex as the reference's reader converts them
(src/basic/io_binary.c:429-500).
"""
from __future__ import annotations

import numpy as np

# type codes of src/basic/io_binary.h:34-40 -> numpy element type
TYPE_FLOAT, TYPE_DOUBLE, TYPE_FLOAT_COMPLEX, TYPE_DOUBLE_COMPLEX, TYPE_INT_32, TYPE_INT_64 = range(6)
_NP_TYPES = {TYPE_FLOAT: "f4", TYPE_DOUBLE: "f8", TYPE_FLOAT_COMPLEX: "c8", TYPE_DOUBLE_COMPLEX: "c16",
             TYPE_INT_32: "i4", TYPE_INT_64: "i8"}
_TYPE_OF = {np.dtype(v): k for k, v in _NP_TYPES.items()}

HEADER = np.dtype([("text", "S7"), ("version", "u1"), ("one_32", "<u4"), ("one_f", "<f4"),
                   ("one_64", "<u8"), ("one_d", "<f8"), ("np", "<u8"), ("type", "<u4"),
                   ("extra", "<u4", (5,))])
assert HEADER.itemsize == 64


def write_obf(path, values) -> None:
    """Write a 1-D array (float32/64, complex64/128, int32/64) as the
    reference's write_binary does (header, then the values, native
    little-endian)."""
    v = np.ascontiguousarray(values)
    if v.ndim != 1 or v.dtype not in _TYPE_OF:
        raise ValueError("write_obf: need a 1-D float, complex or int array")
    if v.shape[0] < 1:
        raise ValueError("write_obf: the reference's format needs at least one value")
    h = np.zeros((), dtype=HEADER)
    h["text"] = b"pulpo"
    h["one_32"], h["one_f"], h["one_64"], h["one_d"] = 1, 1.0, 1, 1.0
    h["np"] = v.shape[0]
    h["type"] = _TYPE_OF[v.dtype]
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(v.astype(v.dtype.newbyteorder("<")).tobytes())


def read_obf(path) -> np.ndarray:
    """Values of an .obf file in their stored type (native byte order),
    with the header checks of check_header (src/basic/io_binary.c:152-192):
    text, version, byte order from the stored one; byte-swapped files are
    converted."""
    with open(path, "rb") as f:
        raw = f.read()
    if len(raw) < 64:
        raise ValueError(f"{path}: file shorter than its header")
    h = np.frombuffer(raw[:64], dtype=HEADER)[0]
    if bytes(h["text"]).rstrip(b"\0") != b"pulpo" or int(h["version"]) != 0:
        raise ValueError(f"{path}: not an io_binary file (text or version)")
    if int(h["one_32"]) == 1:
        end = "<"
    elif int(h["one_32"]) == 1 << 24:
        end = ">"
        h = np.frombuffer(raw[:64], dtype=HEADER.newbyteorder(">"))[0]
    else:
        raise ValueError(f"{path}: unknown byte order")
    n, typ = int(h["np"]), int(h["type"])
    if typ not in _NP_TYPES:
        raise ValueError(f"{path}: unknown payload type {typ}")
    dt = np.dtype(end + _NP_TYPES[typ])
    if len(raw) < 64 + n * dt.itemsize:
        raise ValueError(f"{path}: file shorter than its {n} values")
    return np.frombuffer(raw[64: 64 + n * dt.itemsize], dtype=dt).astype(dt.newbyteorder("="))


def load_states_obf(paths, mesh, ld=None, dtype=np.complex128) -> np.ndarray:
    """A packed (np_part, ld) batch from one .obf file per state (each with
    the mesh's np inner points in mesh order): state i in column i, boundary
    rows and columns past the states zero.  Real files become complex with
    zero imaginary part."""
    paths = list(paths)
    ld = len(paths) if ld is None else int(ld)
    if ld < len(paths):
        raise ValueError("load_states_obf: ld smaller than the number of states")
    out = np.zeros((mesh.np_part, ld), dtype=dtype)
    for i, p in enumerate(paths):
        v = read_obf(p)
        if v.dtype.kind not in "fc":
            raise ValueError(f"{p}: not a mesh function (integer payload)")
        if v.shape[0] != mesh.np:
            raise ValueError(f"{p}: holds {v.shape[0]} points, the mesh has {mesh.np} inner points")
        out[: mesh.np, i] = v
    return out


def save_states_obf(batch, mesh, paths) -> None:
    """One .obf file per state from a packed (npts, ld) batch (numpy or a
    torch tensor, device tensors copied to the host): column i, inner rows
    only, as the reference writes a state for a restart
    (X(restart_write_mesh_function), src/grid/restart_inc.F90:21-97), so a
    reference run can continue from states this library propagated."""
    paths = list(paths)
    try:
        import torch
        if isinstance(batch, torch.Tensor):
            batch = batch.detach().cpu().numpy()
    except ImportError:  # pragma: no cover
        pass
    b = np.asarray(batch)
    if b.ndim != 2 or b.shape[0] < mesh.np or b.shape[1] < len(paths):
        raise ValueError("save_states_obf: batch must be (>= np, >= number of files)")
    for i, p in enumerate(paths):
        write_obf(p, np.ascontiguousarray(b[: mesh.np, i]))
