"""ctypes binding of libhpsi.so (the C ABI declared in include/hpsi.h).

This is the Python host's counterpart of the Fortran ``bind(C)`` interface a
maintainer adds to Octopus: the same entry points, the same argument meaning,
and errors raised from the library's status codes.  Batches are torch tensors
(device memory, streams) or numpy arrays (host memory, staged by the
library).  There is no CPU fallback: if the shared library is missing the
import fails.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "libhpsi.so")

HPSI_C128 = 0
HPSI_C64 = 1
TERM_KINETIC = 1
TERM_LOCAL_POTENTIAL = 2
TERM_NON_LOCAL_POTENTIAL = 4
TERM_ALL = 0x7FFFFFFF
POINTS_ALL = 0
POINTS_INNER = 1
POINTS_OUTER = 2

STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_INDEX", 3: "ERR_NONFINITE", 4: "ERR_CUDA", 5: "ERR_TIMEOUT",
          6: "ERR_STATE", 7: "ERR_NOMEM", 8: "ERR_RUNAWAY", 9: "ERR_UNSUPPORTED"}


class HpsiError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class MeshDesc(C.Structure):
    _fields_ = [("np", C.c_int32), ("np_part", C.c_int32), ("lxyz", C.POINTER(C.c_int32)),
                ("spacing", C.c_double * 3), ("order", C.c_int32), ("periodic", C.c_int32),
                ("per_inner", C.POINTER(C.c_int32))]


class Laser(C.Structure):
    _fields_ = [("E0", C.c_double), ("omega", C.c_double), ("T", C.c_double), ("pol", C.c_double * 3)]


class Batch(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("ld", C.c_int64), ("nst", C.c_int32), ("npts", C.c_int32),
                ("dtype", C.c_int32)]


_lib = None

# declared entry points: name -> (restype, argtypes)
SIGNATURES = {
    "hpsi_mesh_create": (C.c_int32, [C.POINTER(MeshDesc), C.POINTER(C.c_void_p)]),
    "hpsi_mesh_destroy": (C.c_int32, [C.c_void_p]),
    "hpsi_mesh_info": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int32)]),
    "hpsi_hamiltonian_create": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "hpsi_hamiltonian_destroy": (C.c_int32, [C.c_void_p]),
    "hpsi_hamiltonian_set_kinetic": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32),
                                                 C.POINTER(C.c_double), C.c_double]),
    "hpsi_hamiltonian_set_vloc": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double)]),
    "hpsi_hamiltonian_update_vloc": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "hpsi_hamiltonian_set_field": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double), C.c_double]),
    "hpsi_hamiltonian_set_phase_corr": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double)]),
    "hpsi_hamiltonian_set_projectors": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32),
                                                    C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                                    C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "hpsi_hamiltonian_set_projector_phases": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double), C.c_int32]),
    "hpsi_apply_h": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.POINTER(Batch), C.c_int32, C.c_int32,
                                 C.c_void_p]),
    "hpsi_boundaries_set": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.c_void_p]),
    "hpsi_taylor_step": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.c_double, C.c_double, C.c_int32,
                                     C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                     C.c_void_p]),
    "hpsi_td_propagate": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.c_int32, C.c_double, C.c_int32,
                                      C.POINTER(Laser), C.c_double, C.c_int32, C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p]),
    "hpsi_td_propagate_etrs": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.c_int32, C.c_double, C.c_int32,
                                           C.POINTER(Laser), C.c_double, C.c_int32, C.POINTER(C.c_double),
                                           C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p]),
    "hpsi_lanczos_step": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.c_double, C.c_int32, C.c_double,
                                      C.POINTER(C.c_int32), C.POINTER(C.c_double), C.c_void_p]),
    "hpsi_taylor_step_density": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.c_double, C.c_double, C.c_int32,
                                             C.POINTER(C.c_double), C.c_void_p, C.c_int32, C.c_void_p]),
    "hpsi_taylor_step_dual": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.POINTER(Batch), C.c_double, C.c_double,
                                          C.c_double, C.c_double, C.c_int32, C.c_void_p]),
    "hpsi_ghost_pack": (C.c_int32, [C.POINTER(Batch), C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "hpsi_ghost_unpack": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(Batch), C.c_void_p]),
    "hpsi_projector_count": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int32)]),
    "hpsi_projector_bra": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.c_void_p, C.c_void_p]),
    "hpsi_projector_ket": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.POINTER(Batch),
                                       C.c_void_p]),
    "hpsi_apply_h_horner": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.POINTER(Batch), C.POINTER(Batch),
                                        C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_void_p]),
    "hpsi_hamiltonian_status": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int32)]),
    "hpsi_mesh_set_ghost_rows": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32]),
    "hpsi_apply_h_points": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.POINTER(Batch), C.c_int32, C.c_int32,
                                        C.c_int32, C.c_void_p]),
    "hpsi_apply_h_horner_points": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.POINTER(Batch), C.POINTER(Batch),
                                               C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_int32,
                                               C.c_void_p]),
    "hpsi_group_create": (C.c_int32, [C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "hpsi_group_destroy": (C.c_int32, [C.c_void_p]),
    "hpsi_group_taylor_steps": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.c_int32, C.c_double, C.c_int32,
                                            C.c_int32, C.c_void_p]),
    "hpsi_autotune": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                  C.c_void_p]),
    "hpsi_adjoint_gradient": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.POINTER(Batch), C.c_int32, C.c_double,
                                          C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int32,
                                          C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double), C.c_void_p]),
    "hpsi_adjoint_step": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.POINTER(Batch), C.c_double,
                                      C.POINTER(C.c_double), C.c_double, C.c_int32, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]),
    "hpsi_vjp_field": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.POINTER(Batch), C.POINTER(C.c_double),
                                   C.c_void_p, C.c_void_p]),
    "hpsi_vjp_vloc": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.POINTER(Batch), C.c_double, C.c_void_p,
                                  C.c_int32, C.c_void_p]),
    "hpsi_nrm2": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.POINTER(C.c_double), C.c_void_p]),
    "hpsi_density_accumulate": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.POINTER(C.c_double), C.c_void_p,
                                            C.c_int32, C.c_void_p]),
    "hpsi_dotp_matrix": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.POINTER(Batch), C.POINTER(C.c_double),
                                     C.c_void_p]),
    "hpsi_orthonormalize_cholesky": (C.c_int32, [C.c_void_p, C.POINTER(Batch), C.c_void_p]),
    "hpsi_last_error_string": (C.c_char_p, []),
    "hpsi_kernel_launch_count": (C.c_int64, []),
    "hpsi_version": (C.c_char_p, []),
    "hpsi_nrm2_noalloc": (C.c_int32, [C.c_int32, C.c_double, C.POINTER(Batch), C.POINTER(C.c_double),
                                      C.c_void_p]),
    "hpsi_profile_enable": (C.c_int32, [C.c_int32]),
    "hpsi_profile_query": (C.c_int32, [C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_double)]),
}


def load():
    """Load libhpsi.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not built (run `make` in {PKG})")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status: int):
    if status != 0:
        raise HpsiError(status, load().hpsi_last_error_string().decode())


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _stream_ptr(stream):
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available():
                return C.c_void_p(torch.cuda.current_stream().cuda_stream)
        except Exception:  # pragma: no cover
            pass
        return None
    return C.c_void_p(getattr(stream, "cuda_stream", stream))


def as_batch(x, npts=None, nst=None) -> Batch:
    """Describe a packed batch: a (npts, ld) complex torch tensor or numpy array."""
    b = Batch()
    try:
        import torch
        is_t = isinstance(x, torch.Tensor)
    except ImportError:  # pragma: no cover
        is_t = False
    if is_t:
        if x.dim() != 2 or not x.is_contiguous():
            raise ValueError("batch must be a contiguous (npts, ld) tensor")
        if x.dtype == torch.complex128:
            b.dtype = HPSI_C128
        elif x.dtype == torch.complex64:
            b.dtype = HPSI_C64
        else:
            raise ValueError("batch dtype must be complex128 or complex64")
        b.ptr = x.data_ptr()
    else:
        x = np.asarray(x)
        if x.ndim != 2 or not x.flags.c_contiguous:
            raise ValueError("batch must be a C-contiguous (npts, ld) array")
        b.dtype = {np.dtype(np.complex128): HPSI_C128, np.dtype(np.complex64): HPSI_C64}[x.dtype]
        b.ptr = x.ctypes.data
    b.ld = x.shape[1]
    b.npts = x.shape[0] if npts is None else npts
    b.nst = x.shape[1] if nst is None else nst
    return b


class DeviceMesh:
    """hpsi_mesh handle built from a host :class:`hpsi.mesh.Mesh`."""

    def __init__(self, mesh, order: int = 4):
        L = load()
        self.mesh = mesh
        self._lxyz = np.ascontiguousarray(mesh.lxyz.astype(np.int32))
        d = MeshDesc()
        d.np = mesh.np
        d.np_part = mesh.np_part
        d.lxyz = _ip(self._lxyz)
        for a in range(3):
            d.spacing[a] = float(mesh.spacing[a])
        d.order = order
        d.periodic = 1 if mesh.periodic else 0
        self._per = None
        if mesh.periodic:
            self._per = np.ascontiguousarray(mesh.per_inner.astype(np.int32))
            d.per_inner = _ip(self._per)
        h = C.c_void_p()
        check(L.hpsi_mesh_create(C.byref(d), C.byref(h)))
        self.handle = h

    def set_ghost_rows(self, first: int, count: int):
        """Rows [first, first + count) are ghost rows (domain-parallel mesh)."""
        check(load().hpsi_mesh_set_ghost_rows(self.handle, int(first), int(count)))

    def info(self):
        dims = (C.c_int32 * 6)()
        check(load().hpsi_mesh_info(self.handle, dims))
        return list(dims)

    def close(self):
        if getattr(self, "handle", None):
            load().hpsi_mesh_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # reductions (mesh_batch_* of the reference)
    def nrm2(self, psi, nst=None, stream=None) -> np.ndarray:
        b = as_batch(psi, nst=nst)
        out = np.zeros(b.nst)
        check(load().hpsi_nrm2(self.handle, C.byref(b), _dp(out), _stream_ptr(stream)))
        return out

    def density(self, psi, weight, rho=None, accumulate=False, nst=None, stream=None):
        """rho (+)= sum_i weight[i] |psi_i|^2 on the inner points (density_calc_accumulate);
        rho: a float64 device tensor of np entries (allocated when None)."""
        import torch
        b = as_batch(psi, nst=nst)
        w = np.ascontiguousarray(np.asarray(weight, dtype=np.float64)[: b.nst])
        if rho is None:
            rho = torch.zeros(self.mesh.np, dtype=torch.float64, device=psi.device)
        check(load().hpsi_density_accumulate(self.handle, C.byref(b), _dp(w), C.c_void_p(rho.data_ptr()),
                                             1 if accumulate else 0, _stream_ptr(stream)))
        return rho

    def dotp_matrix(self, a, b, nst=None, stream=None) -> np.ndarray:
        ba, bb = as_batch(a, nst=nst), as_batch(b, nst=nst)
        out = np.zeros((ba.nst, ba.nst), dtype=np.complex128)
        check(load().hpsi_dotp_matrix(self.handle, C.byref(ba), C.byref(bb), _dp(out.view(np.float64)),
                                      _stream_ptr(stream)))
        return out

    def orthonormalize_cholesky(self, psi, nst=None, stream=None):
        b = as_batch(psi, nst=nst)
        check(load().hpsi_orthonormalize_cholesky(self.handle, C.byref(b), _stream_ptr(stream)))


class Hamiltonian:
    """hpsi_hamiltonian handle: kinetic weights, local potential, KB projectors."""

    def __init__(self, dmesh: DeviceMesh, weights, points, v=None, projectors=None, factor=-0.5):
        L = load()
        self.dmesh = dmesh
        h = C.c_void_p()
        check(L.hpsi_hamiltonian_create(dmesh.handle, C.byref(h)))
        self.handle = h
        pts = np.ascontiguousarray(np.asarray(points, dtype=np.int32))
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
        check(L.hpsi_hamiltonian_set_kinetic(h, len(w), _ip(pts), _dp(w), C.c_double(factor)))
        if v is not None:
            self.set_vloc(v)
        if projectors is not None:
            self.set_projectors(projectors.maps, projectors.mats, projectors.scals)

    def set_vloc(self, v):
        v = np.ascontiguousarray(np.asarray(v, dtype=np.float64))
        check(load().hpsi_hamiltonian_set_vloc(self.handle, _dp(v)))

    def update_vloc(self, v, stream=None):
        """Stream-ordered potential update (hpsi_hamiltonian_update_vloc): ``v``
        a float64 device tensor of np entries, or a host array."""
        try:
            import torch
            if isinstance(v, torch.Tensor):
                if v.dtype != torch.float64 or not v.is_contiguous() or v.numel() < self.dmesh.mesh.np:
                    raise ValueError("update_vloc: contiguous float64 tensor of np entries expected")
                ptr = C.c_void_p(v.data_ptr())
                check(load().hpsi_hamiltonian_update_vloc(self.handle, ptr, _stream_ptr(stream)))
                return
        except ImportError:  # pragma: no cover
            pass
        v = np.ascontiguousarray(np.asarray(v, dtype=np.float64))
        if v.size < self.dmesh.mesh.np:
            raise ValueError("update_vloc: np entries expected")
        self._vhost = v  # kept alive until the next update (pinned copies read it later)
        check(load().hpsi_hamiltonian_update_vloc(self.handle, C.c_void_p(v.ctypes.data), _stream_ptr(stream)))

    def set_field(self, pol, amplitude: float):
        p = np.ascontiguousarray(np.asarray(pol, dtype=np.float64))
        check(load().hpsi_hamiltonian_set_field(self.handle, _dp(p), C.c_double(amplitude)))

    def set_phase_corr(self, phase_corr):
        if phase_corr is None:
            check(load().hpsi_hamiltonian_set_phase_corr(self.handle, None))
            return
        pc = np.ascontiguousarray(np.asarray(phase_corr, dtype=np.complex128))
        check(load().hpsi_hamiltonian_set_phase_corr(self.handle, _dp(pc.view(np.float64))))

    def set_projectors(self, maps, mats, scals):
        npts = np.asarray([len(m) for m in maps], dtype=np.int32)
        nproj = np.asarray([m.shape[1] for m in mats], dtype=np.int32)
        mp = np.ascontiguousarray(np.concatenate(maps).astype(np.int32))
        mt = np.ascontiguousarray(np.concatenate([np.asarray(m, dtype=np.float64).T.ravel() for m in mats]))
        sc = np.ascontiguousarray(np.concatenate(scals).astype(np.float64))
        check(load().hpsi_hamiltonian_set_projectors(self.handle, len(maps), _ip(npts), _ip(nproj), _ip(mp),
                                                     _dp(mt), _dp(sc)))
        self._kb_npoints = [int(n) for n in npts]

    def set_projector_phases(self, phases, ld_points=0):
        """Per sphere point complex phases: a list with one array per matrix,
        one concatenated array (ld_points = 0), or a padded (nmat, ld_points)
        array / its flattening (point k of matrix m at m * ld_points + k, the
        reference's projector_phases(:, 1, :, ik)); None removes them."""
        if phases is None:
            check(load().hpsi_hamiltonian_set_projector_phases(self.handle, None, 0))
            return
        npts = getattr(self, "_kb_npoints", None)
        if npts is None:
            raise ValueError("set_projector_phases: no projectors set")
        if isinstance(phases, (list, tuple)):
            if [len(a) for a in phases] != list(npts):
                raise ValueError("set_projector_phases: one phase per sphere point of each matrix expected")
            phases = np.concatenate([np.asarray(a, dtype=np.complex128) for a in phases])
            ld_points = 0
        ph = np.ascontiguousarray(np.asarray(phases, dtype=np.complex128)).ravel()
        need = sum(npts) if ld_points == 0 else len(npts) * int(ld_points)
        if ld_points and ld_points < max(npts):
            raise ValueError(f"set_projector_phases: ld_points {ld_points} below the largest sphere ({max(npts)})")
        if ph.size != need:
            raise ValueError(f"set_projector_phases: {ph.size} phases given, {need} expected")
        check(load().hpsi_hamiltonian_set_projector_phases(self.handle, _dp(ph.view(np.float64)), int(ld_points)))

    def autotune(self, dtype=HPSI_C128, ld=32, stream=None):
        """Pick the fastest pass shape for batches of width ld; returns
        ({sc, ry, zb, tile}, ms)."""
        shp = (C.c_int32 * 4)()
        ms = C.c_double()
        check(load().hpsi_autotune(self.handle, int(dtype), int(ld), shp, C.byref(ms), _stream_ptr(stream)))
        return dict(sc=shp[0], ry=shp[1], zb=shp[2], tile=shp[3]), float(ms.value)

    def adjoint_gradient(self, psi0, targets, eps, dt, order=4, pol=(0.0, 0.0, 1.0), ckpt=25, want_v=True,
                         stream=None):
        """(J, dJ/deps, dJ/dv or None, continuous-adjoint dJ/deps) for J = sum |<phi|psi(T)>|^2."""
        eps = np.ascontiguousarray(np.asarray(eps, dtype=np.float64))
        n = len(eps)
        b0, bt = as_batch(psi0), as_batch(targets)
        p = np.ascontiguousarray(np.asarray(pol, dtype=np.float64))
        J = C.c_double()
        ge, gc = np.zeros(n), np.zeros(n)
        gv = np.zeros(self.dmesh.mesh.np) if want_v else None
        check(load().hpsi_adjoint_gradient(self.handle, C.byref(b0), C.byref(bt), n, float(dt), int(order), _dp(eps),
                                           _dp(p), int(ckpt), C.byref(J), _dp(ge), _dp(gv) if want_v else None,
                                           _dp(gc), _stream_ptr(stream)))
        return float(J.value), ge, gv, gc

    # per-step adjoint primitives (host-driven backward propagation)
    def adjoint_step(self, lam, psi_n, eps_n, dt, order=4, pol=(0.0, 0.0, 1.0), grad_v=None, stream=None):
        """lam <- T_n^dagger lam in place; returns (dJ/d eps_n, continuous-adjoint
        term) and accumulates dJ/dv into the float64 device tensor grad_v."""
        bl, bp = as_batch(lam), as_batch(psi_n)
        p = np.ascontiguousarray(np.asarray(pol, dtype=np.float64))
        ge, gc = np.zeros(1), np.zeros(1)
        gv = C.c_void_p(grad_v.data_ptr()) if grad_v is not None else None
        check(load().hpsi_adjoint_step(self.handle, C.byref(bl), C.byref(bp), float(eps_n), _dp(p), float(dt),
                                       int(order), C.c_void_p(ge.ctypes.data), C.c_void_p(gc.ctypes.data), gv,
                                       _stream_ptr(stream)))
        return float(ge[0]), float(gc[0])

    def vjp_field(self, chi, psi, pol=(0.0, 0.0, 1.0), nst=None, stream=None) -> np.ndarray:
        """Per-state dV <chi_i|pol.r|psi_i> (complex, host array)."""
        bc, bp = as_batch(chi, nst=nst), as_batch(psi, nst=nst)
        p = np.ascontiguousarray(np.asarray(pol, dtype=np.float64))
        out = np.zeros(bc.nst, dtype=np.complex128)
        check(load().hpsi_vjp_field(self.handle, C.byref(bc), C.byref(bp), _dp(p),
                                    C.c_void_p(out.ctypes.data), _stream_ptr(stream)))
        return out

    def vjp_vloc(self, lam, psi, grad_v, scale=1.0, accumulate=False, nst=None, stream=None):
        """grad_v (+)= scale sum_i Re(conj(lam_i) psi_i) on the inner rows
        (float64 device tensor of np entries)."""
        bl, bp = as_batch(lam, nst=nst), as_batch(psi, nst=nst)
        check(load().hpsi_vjp_vloc(self.handle, C.byref(bl), C.byref(bp), float(scale),
                                   C.c_void_p(grad_v.data_ptr()), 1 if accumulate else 0, _stream_ptr(stream)))
        return grad_v

    # exponential-midpoint time propagation (td_run with TDPropagator = exp_mid)
    def td_propagate(self, psi, nsteps, dt, order=4, E0=0.0, omega=0.0, T=0.0, pol=(0.0, 0.0, 1.0), t0=0.0,
                     graph=True, nst=None, stream=None, propagator="exp_mid"):
        """propagator: "exp_mid" (hpsi_td_propagate) or "etrs" (hpsi_td_propagate_etrs)."""
        b = as_batch(psi, nst=nst)
        las = Laser()
        las.E0, las.omega, las.T = float(E0), float(omega), float(T)
        for a in range(3):
            las.pol[a] = float(pol[a])
        e, d, n = np.zeros(nsteps), np.zeros(nsteps), np.zeros(nsteps)
        fn = {"exp_mid": load().hpsi_td_propagate, "etrs": load().hpsi_td_propagate_etrs}[propagator]
        check(fn(self.handle, C.byref(b), int(nsteps), float(dt), int(order), C.byref(las), float(t0),
                 1 if graph else 0, _dp(e), _dp(d), _dp(n), _stream_ptr(stream)))
        return e, d, n

    def close(self):
        if getattr(self, "handle", None):
            load().hpsi_hamiltonian_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # X(hamiltonian_elec_apply_batch)
    def apply(self, psi, hpsi, nst=None, terms=TERM_ALL, set_bc=True, stream=None, points=POINTS_ALL):
        """points: POINTS_ALL, or POINTS_INNER / POINTS_OUTER on a mesh with
        ghost rows (hpsi_apply_h_points)."""
        bi = as_batch(psi, nst=nst)
        bo = as_batch(hpsi, nst=nst)
        if points == POINTS_ALL:
            check(load().hpsi_apply_h(self.handle, C.byref(bi), C.byref(bo), terms, 1 if set_bc else 0,
                                      _stream_ptr(stream)))
        else:
            check(load().hpsi_apply_h_points(self.handle, C.byref(bi), C.byref(bo), terms, 1 if set_bc else 0,
                                             int(points), _stream_ptr(stream)))

    def status(self) -> int:
        """Status word of the bounded waits of this Hamiltonian's passes
        (hpsi_hamiltonian_status: 0, or 5 = HPSI_ERR_TIMEOUT); clears it."""
        st = C.c_int32()
        check(load().hpsi_hamiltonian_status(self.handle, C.byref(st)))
        return int(st.value)

    def nprojections(self) -> int:
        n = C.c_int32()
        check(load().hpsi_projector_count(self.handle, C.byref(n)))
        return int(n.value)

    # X(hamiltonian_elec_base_nlocal_start), without the reduction
    def projector_bra(self, psi, proj, stream=None):
        """proj (nprojections, ld) <- the KB projections of the device batch
        psi (hpsi_projector_bra)."""
        b = as_batch(psi)
        check(load().hpsi_projector_bra(self.handle, C.byref(b), C.c_void_p(proj.data_ptr()),
                                        _stream_ptr(stream)))

    # X(hamiltonian_elec_base_nlocal_finish), after the reduction
    def projector_ket(self, proj, hpsi, nst=None, a=1.0, stream=None):
        """hpsi += a P proj on the covered rows (hpsi_projector_ket)."""
        b = as_batch(hpsi, nst=nst)
        a = complex(a)
        check(load().hpsi_projector_ket(self.handle, C.c_void_p(proj.data_ptr()), a.real, a.imag, C.byref(b),
                                        _stream_ptr(stream)))

    def apply_horner(self, psi, psi0, out, a, nst=None, terms=TERM_ALL, set_bc=True, stream=None,
                     points=POINTS_ALL):
        """out = psi0 + a H psi on the inner rows (hpsi_apply_h_horner; with
        points INNER / OUTER the part of hpsi_apply_h_horner_points)."""
        bi, b0, bo = as_batch(psi, nst=nst), as_batch(psi0, nst=nst), as_batch(out, nst=nst)
        a = complex(a)
        if points == POINTS_ALL:
            check(load().hpsi_apply_h_horner(self.handle, C.byref(bi), C.byref(b0), C.byref(bo), a.real, a.imag,
                                             terms, 1 if set_bc else 0, _stream_ptr(stream)))
        else:
            check(load().hpsi_apply_h_horner_points(self.handle, C.byref(bi), C.byref(b0), C.byref(bo), a.real,
                                                    a.imag, terms, 1 if set_bc else 0, int(points),
                                                    _stream_ptr(stream)))

    def boundaries_set(self, psi, nst=None, stream=None):
        b = as_batch(psi, nst=nst)
        check(load().hpsi_boundaries_set(self.handle, C.byref(b), _stream_ptr(stream)))

    def taylor_step_dual(self, psi, psi2, dt, dt2, order=4, nst=None, stream=None):
        """psi2 <- exp(-i dt2 H) psi and psi <- exp(-i dt H) psi (Taylor, the
        psib2 output of exponential_apply_batch)."""
        b, b2 = as_batch(psi, nst=nst), as_batch(psi2, nst=nst)
        dt, dt2 = complex(dt), complex(dt2)
        check(load().hpsi_taylor_step_dual(self.handle, C.byref(b), C.byref(b2), dt.real, dt.imag, dt2.real,
                                           dt2.imag, int(order), _stream_ptr(stream)))

    # Lanczos branch of exponential_apply_batch
    def lanczos_step(self, psi, dt, max_order=30, tol=1e-5, nst=None, stream=None):
        """psi <- exp(-i dt H) psi by Lanczos; returns (Krylov dimension, error estimate)."""
        b = as_batch(psi, nst=nst)
        it = C.c_int32()
        res = C.c_double()
        check(load().hpsi_lanczos_step(self.handle, C.byref(b), float(dt), int(max_order), float(tol), C.byref(it),
                                       C.byref(res), _stream_ptr(stream)))
        return int(it.value), float(res.value)

    def taylor_step_density(self, psi, dt, weight, rho=None, accumulate=False, order=4, nst=None, stream=None):
        """Taylor step, then rho (+)= sum_i weight[i] |psi_i|^2 of the propagated
        batch, fused into the last pass (hpsi_taylor_step_density); rho a
        float64 device tensor of np entries (allocated when None)."""
        import torch
        b = as_batch(psi, nst=nst)
        w = np.ascontiguousarray(np.asarray(weight, dtype=np.float64)[: b.nst])
        if rho is None:
            rho = torch.zeros(self.dmesh.mesh.np, dtype=torch.float64, device=psi.device)
        dt = complex(dt)
        check(load().hpsi_taylor_step_density(self.handle, C.byref(b), dt.real, dt.imag, int(order), _dp(w),
                                              C.c_void_p(rho.data_ptr()), 1 if accumulate else 0,
                                              _stream_ptr(stream)))
        return rho

    # Taylor branch of exponential_apply_batch
    def taylor_step(self, psi, dt, order=4, nst=None, observables=False, stream=None):
        b = as_batch(psi, nst=nst)
        dt = complex(dt)
        if observables:
            e, d, n = np.zeros(b.nst), np.zeros(b.nst), np.zeros(b.nst)
            check(load().hpsi_taylor_step(self.handle, C.byref(b), dt.real, dt.imag, order, _dp(e), _dp(d),
                                          _dp(n), _stream_ptr(stream)))
            return e, d, n
        check(load().hpsi_taylor_step(self.handle, C.byref(b), dt.real, dt.imag, order, None, None, None,
                                      _stream_ptr(stream)))
        return None


class Group:
    """Independent systems advanced together (hpsi_group)."""

    def __init__(self, hams):
        self.hams = list(hams)
        arr = (C.c_void_p * len(self.hams))(*[h.handle.value for h in self.hams])
        h = C.c_void_p()
        check(load().hpsi_group_create(len(self.hams), arr, C.byref(h)))
        self.handle = h

    def taylor_steps(self, psis, nsteps, dt, order=4, graph=True, nsts=None, stream=None):
        bs = (Batch * len(psis))()
        for i, x in enumerate(psis):
            bs[i] = as_batch(x, nst=None if nsts is None else nsts[i])
        check(load().hpsi_group_taylor_steps(self.handle, bs, int(nsteps), float(dt), int(order), 1 if graph else 0,
                                             _stream_ptr(stream)))

    def close(self):
        if getattr(self, "handle", None):
            load().hpsi_group_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def nrm2_noalloc(np_inner: int, vol_pp: float, psi, nst=None, stream=None) -> np.ndarray:
    """State norms through the allocation-free entry point (host result)."""
    b = as_batch(psi, nst=nst)
    out = np.zeros(b.nst)
    check(load().hpsi_nrm2_noalloc(int(np_inner), float(vol_pp), C.byref(b), _dp(out), _stream_ptr(stream)))
    return out


def launch_count() -> int:
    return int(load().hpsi_kernel_launch_count())


def profile_enable(on: bool = True):
    check(load().hpsi_profile_enable(1 if on else 0))


def profile_query(label: str):
    """(launches, total device ms) of one kernel label since profile_enable."""
    n = C.c_int64()
    ms = C.c_double()
    check(load().hpsi_profile_query(label.encode(), C.byref(n), C.byref(ms)))
    return int(n.value), float(ms.value)


def ghost_pack(psi, sendmap, out, nst=None, stream=None):
    """out[i, :nst] = psi[sendmap[i], :nst] on the device (hpsi_ghost_pack).

    ``sendmap`` an int32 device tensor, ``out`` a contiguous (count, nst) device
    tensor of psi's dtype."""
    b = as_batch(psi, nst=nst)
    check(load().hpsi_ghost_pack(C.byref(b), sendmap.data_ptr(), int(sendmap.numel()), out.data_ptr(),
                                 _stream_ptr(stream)))


def ghost_unpack(buf, pos, psi, nst=None, stream=None):
    """psi[pos[i], :nst] = buf[i, :nst] on the device (hpsi_ghost_unpack)."""
    b = as_batch(psi, nst=nst)
    check(load().hpsi_ghost_unpack(buf.data_ptr(), pos.data_ptr(), int(pos.numel()), C.byref(b),
                                   _stream_ptr(stream)))
