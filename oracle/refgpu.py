"""The reference's own GPU H.psi, for comparison only (test infrastructure).

Loads the CUBINs oracle/refgpu_build.py compiled from the reference's
share/opencl kernels and launches them in the order and with the launch
geometry of the reference's CUDA path of X(hamiltonian_elec_apply_batch)
(src/hamiltonian/hamiltonian_elec_inc.F90:77-261) for a real-projector,
zero-boundary, unpolarised batch, on the packed batch viewed as reals
(pack_size_real = 2 * pack_size, powers of two as batch_t pads them):

1. kinetic: operate_map with the weights times -1/2
   (X(nl_operator_operate_batch) OP_MAP branch, src/grid/nl_operator_inc.F90:316-379:
   global (eff_size, dim2, dim3), local (eff_size, localsize), dynamic shared
   memory localsize * STENCIL_SIZE ints);
2. local potential: vpsi (src/hamiltonian/hamiltonian_elec_base_inc.F90:118-135);
3. KB bra: dprojector_bra, global (size * warp, pad_pow2(max nprojs), nmat),
   local (warp, min(1024 / warp, pad_pow2(max nprojs))) (:548-592);
4. KB ket: dprojector_ket once per matrix, each launch followed by a device
   synchronisation (accel_finish) (:1125-1180).
and daxpy (axpy.cl:26-35, a real factor on the real view: the real-factor
terms of exponential_taylor_series_batch, src/electrons/exponential.F90:738-744).

Nothing in the library imports this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")
WARP = 32
MAX_WG = 1024            # accel%max_workgroup_size (threads per block)
MAX_DIM2 = 32768         # accel_max_size_per_dim(2)
OFFSET_SIZE = 6          # POINTS, PROJS, MATRIX, MAP, SCAL, MIX


def available() -> bool:
    return all(os.path.exists(os.path.join(REF, f"refcl_{n}.cubin"))
               for n in ("operate", "vpsi", "projector_d", "axpy_d"))


def _pad(n, m):
    return ((n + m - 1) // m) * m


def _pow2(n):
    p = 1
    while p < n:
        p *= 2
    return p


class _Kernels:
    def __init__(self):
        from cuda.bindings import driver as cu
        self.cu = cu
        self.mods = {}
        self.fns = {}
        for unit, names in (("operate", ["operate_map"]), ("vpsi", ["vpsi"]),
                            ("projector_d", ["dprojector_bra", "dprojector_ket"]),
                            ("axpy_d", ["daxpy"])):
            with open(os.path.join(REF, f"refcl_{unit}.cubin"), "rb") as f:
                data = f.read()
            err, mod = cu.cuModuleLoadData(data)
            if err != cu.CUresult.CUDA_SUCCESS:
                raise RuntimeError(f"cuModuleLoadData {unit}: {err}")
            self.mods[unit] = mod
            for n in names:
                err, fn = cu.cuModuleGetFunction(mod, n.encode())
                if err != cu.CUresult.CUDA_SUCCESS:
                    raise RuntimeError(f"cuModuleGetFunction {n}: {err}")
                self.fns[n] = fn

    def launch(self, name, grid, block, shmem, stream, args):
        vals = tuple(a for a, _ in args)
        types = tuple(t for _, t in args)
        err, = self.cu.cuLaunchKernel(self.fns[name], *grid, *block, shmem, stream, (vals, types), 0)
        if err != self.cu.CUresult.CUDA_SUCCESS:
            raise RuntimeError(f"cuLaunchKernel {name}: {err}")


class RefHamiltonian:
    """Device buffers of the reference's GPU H.psi for one mesh, kinetic
    weights, local potential and real KB projectors."""

    def __init__(self, mesh, weights, points, v, projectors, device):
        import torch
        from oracle import oracle as O
        torch.zeros(1, device=device)  # the primary context is current from here on
        self.k = _Kernels()
        self.mesh = mesh
        self.dev = device
        op = O.Operator(mesh, points)
        self.W = op.W
        self.ri = torch.from_numpy(np.ascontiguousarray(op.ri.astype(np.int32))).to(device)
        # operate_map reads ri[map[ip] + j]: map = run index * W (nl_operator.F90:543-544)
        self.map = torch.from_numpy(np.ascontiguousarray((op.rimap * op.W).astype(np.int32))).to(device)
        self.w = torch.from_numpy(np.ascontiguousarray(np.asarray(weights, dtype=np.float64) * -0.5)).to(device)
        self.v = torch.from_numpy(np.ascontiguousarray(np.asarray(v, dtype=np.float64))).to(device)
        self.proj = projectors
        if projectors is not None:
            npts = [len(m) for m in projectors.maps]
            nprj = [m.shape[1] for m in projectors.mats]
            offs, mo, po, so = [], 0, 0, 0
            for a, b in zip(npts, nprj):
                offs += [a, b, mo, po, so, 0]
                mo += a * b
                po += a
                so += b
            self.nmat = len(npts)
            self.max_nprojs = max(nprj)
            self.max_npoints = max(npts)
            self.nprojections = so
            self.npts = npts
            self.offsets = torch.tensor(offs, dtype=torch.int32, device=device)
            mats = np.concatenate([np.asarray(m, dtype=np.float64).T.ravel() for m in projectors.mats])
            self.matrices = torch.from_numpy(np.ascontiguousarray(mats)).to(device)
            maps1 = np.concatenate([np.asarray(m, dtype=np.int64) for m in projectors.maps]) + 1  # 1-based
            self.maps = torch.from_numpy(np.ascontiguousarray(maps1.astype(np.int32))).to(device)
            self.scal = torch.from_numpy(np.ascontiguousarray(np.concatenate(projectors.scals).astype(np.float64))).to(device)

    def _stream(self):
        import torch
        return self.k.cu.CUstream(torch.cuda.current_stream().cuda_stream)

    def kinetic(self, psi, out):
        """out = -1/2 lapl psi on the inner points (operate_map)."""
        size = 2 * psi.shape[1]
        ld = int(np.log2(size))
        np_ = self.mesh.np
        localsize = MAX_WG // size
        dim3 = np_ // (MAX_DIM2 * localsize) + 1
        dim2 = min(MAX_DIM2 * localsize, _pad(np_, localsize))
        p = C.c_void_p
        self.k.launch("operate_map", (1, dim2 // localsize, dim3), (size, localsize, 1),
                      localsize * self.W * 4, self._stream(),
                      [(np_, C.c_int), (self.ri.data_ptr(), p), (self.map.data_ptr(), p), (self.w.data_ptr(), p),
                       (psi.data_ptr(), p), (ld, C.c_int), (out.data_ptr(), p), (ld, C.c_int)])

    def local(self, psi, out):
        """out += v psi (vpsi)."""
        size = 2 * psi.shape[1]
        ld = int(np.log2(size))
        np_ = self.mesh.np
        localsize = MAX_WG // size
        dim3 = np_ // (MAX_DIM2 * localsize) + 1
        dim2 = min(MAX_DIM2 * localsize, _pad(np_, localsize))
        p = C.c_void_p
        self.k.launch("vpsi", (1, dim2 // localsize, dim3), (size, localsize, 1), 0, self._stream(),
                      [(0, C.c_int), (np_, C.c_int), (self.v.data_ptr(), p), (psi.data_ptr(), p), (ld, C.c_int),
                       (out.data_ptr(), p), (ld, C.c_int)])

    def bra(self, psi, projection):
        """projection (nprojections x pack_size_real doubles) <- dprojector_bra."""
        size = 2 * psi.shape[1]
        ld = int(np.log2(size))
        padnprojs = _pow2(self.max_nprojs)
        lnprojs = min(MAX_WG // WARP, padnprojs)
        p = C.c_void_p
        self.k.launch("dprojector_bra", (size, padnprojs // lnprojs, self.nmat), (WARP, lnprojs, 1), 0,
                      self._stream(),
                      [(self.nmat, C.c_int), (self.offsets.data_ptr(), p), (self.matrices.data_ptr(), p),
                       (self.maps.data_ptr(), p), (self.scal.data_ptr(), p), (psi.data_ptr(), p), (ld, C.c_int),
                       (projection.data_ptr(), p), (ld, C.c_int)])

    def ket(self, projection, out, sync=True):
        """out += P projection, one launch per matrix (dprojector_ket), each
        followed by a synchronisation as accel_finish does."""
        import torch
        size = 2 * out.shape[1]
        ld = int(np.log2(size))
        wg = MAX_WG // size
        p = C.c_void_p
        for imat in range(self.nmat):
            self.k.launch("dprojector_ket", (1, _pad(self.max_npoints, wg) // wg, 1), (size, wg, 1), 0,
                          self._stream(),
                          [(self.nmat, C.c_int), (imat, C.c_int), (self.offsets.data_ptr(), p),
                           (self.matrices.data_ptr(), p), (self.maps.data_ptr(), p), (projection.data_ptr(), p),
                           (ld, C.c_int), (out.data_ptr(), p), (ld, C.c_int), (0, C.c_int),
                           (self.npts[imat], C.c_int)])
            if sync:
                torch.cuda.current_stream().synchronize()

    def projection_buffer(self, psi):
        import torch
        return torch.zeros((self.nprojections, 2 * psi.shape[1]), dtype=torch.float64, device=psi.device)

    def apply(self, psi, out, proj=None, sync=True):
        """out = H psi (kinetic, local, KB) on the inner points; psi a complex128
        device batch (np_part x ld, ld a power of two, zero boundary rows)."""
        self.kinetic(psi, out)
        if self.proj is not None:
            proj = self.projection_buffer(psi) if proj is None else proj
            self.bra(psi, proj)
        self.local(psi, out)
        if self.proj is not None:
            self.ket(proj, out, sync=sync)

    def axpy(self, a_real, x, y):
        """y += a x on the inner points with a real factor (daxpy on the real view)."""
        size = 2 * x.shape[1]
        ld = int(np.log2(size))
        np_ = self.mesh.np
        localsize = MAX_WG // size
        dim3 = np_ // (MAX_DIM2 * localsize) + 1
        dim2 = min(MAX_DIM2 * localsize, _pad(np_, localsize))
        p = C.c_void_p
        self.k.launch("daxpy", (1, dim2 // localsize, dim3), (size, localsize, 1), 0, self._stream(),
                      [(np_, C.c_int), (float(a_real), C.c_double), (x.data_ptr(), p), (ld, C.c_int),
                       (y.data_ptr(), p), (ld, C.c_int)])
