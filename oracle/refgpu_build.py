"""Compile the reference's own GPU kernels (share/opencl/*.cl) for sm_100a.

Test infrastructure only (the GPU comparator of the oracle): nothing in the
library links or calls these.  The reference builds its OpenCL-C kernels for
CUDA at run time with NVRTC (src/basic/cuda_low.cc:180-265: the source is
`#include "<file>"`, the options are `--gpu-architecture=compute_XY
--ftz=true --fmad=true -DCUDA -default-device` plus the include path of
share/opencl, `-DSHARED_MEM` (src/basic/accel.F90:1923-1931) and the
kernel's own flags).  This recipe runs the same NVRTC compilation here, ahead
of time, for sm_100a, reading the sources where they lie in the reference
tree, and writes one CUBIN per (file, flags) into oracle/_ref/:

    python oracle/refgpu_build.py <reference source tree>

Kernel flags as the reference passes them:
  operate.cl    -DNDIM=3 -DSTENCIL_SIZE=25   (src/grid/nl_operator.F90:518-527)
  vpsi.cl       (none)                       (src/basic/accel.F90:649)
  projector.cl  -DRTYPE_DOUBLE               (hamiltonian_elec_base_inc.F90:553, 1132)
  axpy.cl       -DRTYPE_DOUBLE               (src/grid/batch_ops_inc.F90:153)
"""
import ctypes as C
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

UNITS = {
    "operate": ("operate.cl", ["-DNDIM=3", "-DSTENCIL_SIZE=25"]),
    "vpsi": ("vpsi.cl", []),
    "projector_d": ("projector.cl", ["-DRTYPE_DOUBLE"]),
    "axpy_d": ("axpy.cl", ["-DRTYPE_DOUBLE"]),
}


def _nvrtc():
    for p in ("/usr/local/cuda/lib64/libnvrtc.so", "libnvrtc.so", "libnvrtc.so.12"):
        try:
            return C.CDLL(p)
        except OSError:
            continue
    raise SystemExit("libnvrtc not found")


def compile_unit(lib, ref, name, fname, flags):
    cl_dir = os.path.join(ref, "share", "opencl")
    src = f'#include "{os.path.join(cl_dir, fname)}"\n'.encode()
    prog = C.c_void_p()
    rc = lib.nvrtcCreateProgram(C.byref(prog), src, b"kernel_include.c", 0, None, None)
    if rc:
        raise SystemExit(f"nvrtcCreateProgram {name}: {rc}")
    opts = ["--gpu-architecture=sm_100a", "--ftz=true", "--fmad=true", "-DCUDA", "-default-device",
            f"-I{cl_dir}/", "-DSHARED_MEM"] + flags
    arr = (C.c_char_p * len(opts))(*[o.encode() for o in opts])
    rc = lib.nvrtcCompileProgram(prog, len(opts), arr)
    n = C.c_size_t()
    lib.nvrtcGetProgramLogSize(prog, C.byref(n))
    log = C.create_string_buffer(n.value)
    lib.nvrtcGetProgramLog(prog, log)
    if rc:
        raise SystemExit(f"nvrtcCompileProgram {name} failed ({rc}):\n{log.value.decode()}")
    lib.nvrtcGetCUBINSize(prog, C.byref(n))
    buf = C.create_string_buffer(n.value)
    lib.nvrtcGetCUBIN(prog, buf)
    lib.nvrtcDestroyProgram(C.byref(prog))
    path = os.path.join(OUT, f"refcl_{name}.cubin")
    with open(path, "wb") as f:
        f.write(buf.raw)
    return path


def main():
    if len(sys.argv) < 2 or not os.path.isdir(os.path.join(sys.argv[1], "share", "opencl")):
        raise SystemExit("usage: refgpu_build.py <reference source tree>")
    os.makedirs(OUT, exist_ok=True)
    lib = _nvrtc()
    for name, (fname, flags) in UNITS.items():
        print("built", compile_unit(lib, sys.argv[1], name, fname, flags))


if __name__ == "__main__":
    main()
