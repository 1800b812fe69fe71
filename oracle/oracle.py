"""CPU ORACLE -- test infrastructure only (never imported by the product).

Python side of the FP64 oracle: it loads ``liboracle.so`` (the C restatement in
``oracle.c``) and, when present, the reference's own compiled stencil kernel
``_ref/libref_operate.so`` (built from src/grid/operate.c by ``make ref``), and
adds the numpy restatements of the small dense pieces:

* ``mesh_batch_nrm2`` -- src/grid/mesh_batch_inc.F90:970-1167 (norm = sqrt(dV *
  sum |psi|^2) over the np inner points);
* ``mesh_batch_dotp_matrix`` -- src/grid/mesh_batch_inc.F90:20-263
  (S_ij = dV * sum conj(a_i) b_j);
* ``cholesky_orthonormalize`` -- states_elec_orthogonalization_full,
  ``cholesky_serial`` branch, src/states/states_elec_calc_inc.F90:66-98
  (S = U^H U, psi <- psi U^-1);
* ``kb_bra`` / ``kb_ket`` -- the KB projections of a batch and their
  scatter-add back, src/hamiltonian/hamiltonian_elec_base_inc.F90:650-780,
  909-1027 (split at the reduction over domains, :836), with optional projector
  phases for k != 0 (:680-701, 934-1025);
* ``derivatives_test_error`` -- src/grid/derivatives_inc.F90:378-492, the
  Laplacian error that testsuite/components/03-derivatives_3d.test pins.

Only tests, the smoke check and the benchmark's CPU legs use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None


def _build_if_missing():
    so = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return so


def lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(_build_if_missing())
        _LIB.orc_nl_operator_build.restype = C.c_int
        _LIB.orc_max_threads.restype = C.c_int
        _LIB.orc_nprojections.restype = C.c_longlong
    return _LIB


def ref_operate():
    """The reference's own ``doperate_ri_vec_`` if it was compiled, else None."""
    global _REF
    if _REF is None:
        so = os.path.join(HERE, "_ref", "libref_operate.so")
        if os.path.exists(so):
            _REF = C.CDLL(so)
        else:
            _REF = False
    return _REF.doperate_ri_vec_ if _REF else None


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


class OrcCtx(C.Structure):
    _fields_ = [
        ("np", C.c_int), ("np_part", C.c_int), ("ld", C.c_int), ("nst", C.c_int),
        ("W", C.c_int), ("wre", C.POINTER(C.c_double)), ("nri", C.c_int),
        ("ri", C.POINTER(C.c_int)), ("imin", C.POINTER(C.c_int)), ("imax", C.POINTER(C.c_int)),
        ("v", C.POINTER(C.c_double)), ("bc", C.c_int),
        ("per_inner", C.POINTER(C.c_int)), ("phase_corr", C.POINTER(C.c_double)),
        ("nmat", C.c_int), ("pm_npoints", C.POINTER(C.c_int)), ("pm_nprojs", C.POINTER(C.c_int)),
        ("pm_map_off", C.POINTER(C.c_longlong)), ("pm_mat_off", C.POINTER(C.c_longlong)),
        ("pm_scal_off", C.POINTER(C.c_longlong)),
        ("pm_map", C.POINTER(C.c_int)), ("pm_mat", C.POINTER(C.c_double)),
        ("pm_scal", C.POINTER(C.c_double)),
        ("nthreads", C.c_int), ("operate", C.c_void_p),
    ]


def neighbour_table(mesh, points) -> np.ndarray:
    """0-based index of inner point i + stencil point j, shape (np, W).

    This is ``mesh_local_index_from_coords`` evaluated for every stencil point
    (src/grid/nl_operator.F90:352-356)."""
    lx = mesh.lxyz.astype(np.int64)
    lo = lx.min(axis=0)
    ext = lx.max(axis=0) - lo + 1
    lut = -np.ones(ext[::-1], dtype=np.int64)
    ii = lx - lo[None, :]
    lut[ii[:, 2], ii[:, 1], ii[:, 0]] = np.arange(mesh.np_part)
    nb = lx[: mesh.np, None, :] + points[None, :, :] - lo[None, None, :]
    idx = lut[nb[..., 2], nb[..., 1], nb[..., 0]]
    if (idx < 0).any():
        raise ValueError("stencil reaches a point outside the mesh")
    return np.ascontiguousarray(idx.astype(np.int32))


class Operator:
    """``nl_operator_t`` of the Laplacian on a mesh (runs built by the oracle)."""

    def __init__(self, mesh, points):
        nbr = neighbour_table(mesh, points)
        W = points.shape[0]
        L = lib()
        nri = L.orc_nl_operator_build(C.c_int(mesh.np), C.c_int(W), _p(nbr, C.c_int), None, None, None)
        self.ri = np.zeros(nri * W, dtype=np.int32)
        self.rimap = np.zeros(mesh.np, dtype=np.int32)
        self.rimap_inv = np.zeros(nri + 1, dtype=np.int32)
        n2 = L.orc_nl_operator_build(C.c_int(mesh.np), C.c_int(W), _p(nbr, C.c_int), _p(self.ri, C.c_int),
                                     _p(self.rimap, C.c_int), _p(self.rimap_inv, C.c_int))
        assert n2 == nri
        self.nri = nri
        self.W = W
        self.imin = np.ascontiguousarray(self.rimap_inv[:-1])
        self.imax = np.ascontiguousarray(self.rimap_inv[1:])


class Projectors:
    """Concatenated KB projector matrices (``projector_matrix_t`` list)."""

    def __init__(self, maps, mats, scals):
        self.npoints = np.asarray([len(m) for m in maps], dtype=np.int32)
        self.nprojs = np.asarray([m.shape[1] for m in mats], dtype=np.int32)
        self.map_off = np.concatenate([[0], np.cumsum(self.npoints)[:-1]]).astype(np.int64)
        self.mat_off = np.concatenate([[0], np.cumsum(self.npoints.astype(np.int64) * self.nprojs)[:-1]]).astype(np.int64)
        self.scal_off = np.concatenate([[0], np.cumsum(self.nprojs)[:-1]]).astype(np.int64)
        self.map = np.ascontiguousarray(np.concatenate(maps).astype(np.int32))
        # point fastest inside each matrix (Fortran dprojectors(npoints, nprojs))
        self.mat = np.ascontiguousarray(np.concatenate([np.asarray(m, dtype=np.float64).T.ravel() for m in mats]))
        self.scal = np.ascontiguousarray(np.concatenate(scals).astype(np.float64))
        self.nmat = len(maps)
        self.nprojections = int(self.nprojs.sum())


class Hamiltonian:
    """FP64 CPU Hamiltonian apply (kinetic + local + KB) on packed batches."""

    def __init__(self, mesh, weights, points, v=None, projectors=None, bc="zero",
                 phase_corr=None, nthreads=None, use_ref=True):
        self.mesh = mesh
        self.op = Operator(mesh, points)
        self.wre = np.ascontiguousarray(np.asarray(weights, dtype=np.float64) * -0.5)
        self.v = None if v is None else np.ascontiguousarray(np.asarray(v, dtype=np.float64))
        self.proj = projectors
        self.bc = {"none": 0, "zero": 1, "periodic": 2}[bc]
        self.per_inner = mesh.per_inner if self.bc == 2 else None
        self.phase_corr = None if phase_corr is None else np.ascontiguousarray(
            np.asarray(phase_corr, dtype=np.complex128)).view(np.float64)
        self.nthreads = nthreads or lib().orc_max_threads()
        self.ref_fn = ref_operate() if use_ref else None
        self.used_reference_kernel = self.ref_fn is not None

    def _ctx(self, ld, nst):
        c = OrcCtx()
        m = self.mesh
        c.np, c.np_part, c.ld, c.nst, c.W = m.np, m.np_part, ld, nst, self.op.W
        c.wre = _p(self.wre)
        c.nri = self.op.nri
        c.ri, c.imin, c.imax = _p(self.op.ri, C.c_int), _p(self.op.imin, C.c_int), _p(self.op.imax, C.c_int)
        c.v = _p(self.v)
        c.bc = self.bc
        c.per_inner = _p(self.per_inner, C.c_int) if self.per_inner is not None else None
        c.phase_corr = _p(self.phase_corr) if self.phase_corr is not None else None
        if self.proj is not None:
            P = self.proj
            c.nmat = P.nmat
            c.pm_npoints, c.pm_nprojs = _p(P.npoints, C.c_int), _p(P.nprojs, C.c_int)
            c.pm_map_off, c.pm_mat_off, c.pm_scal_off = (_p(P.map_off, C.c_longlong), _p(P.mat_off, C.c_longlong),
                                                         _p(P.scal_off, C.c_longlong))
            c.pm_map, c.pm_mat, c.pm_scal = _p(P.map, C.c_int), _p(P.mat), _p(P.scal)
        else:
            c.nmat = 0
        c.nthreads = self.nthreads
        c.operate = C.cast(self.ref_fn, C.c_void_p).value if self.ref_fn is not None else None
        return c

    @staticmethod
    def packed(psi: np.ndarray) -> tuple[np.ndarray, int]:
        """Copy (npts, nst) complex states into a packed (npts, ld) array."""
        nst = psi.shape[1]
        ld = 1 << (nst - 1).bit_length()
        out = np.zeros((psi.shape[0], ld), dtype=np.complex128)
        out[:, :nst] = psi
        return out, ld

    def apply(self, psi: np.ndarray) -> np.ndarray:
        """H psi for psi of shape (np_part, nst) complex128.  Returns (np, nst).

        The boundary region of the packed copy is set as the reference's
        ``boundaries_set`` does; the caller's array is not modified."""
        m = self.mesh
        nst = psi.shape[1]
        x, ld = self.packed(np.asarray(psi, dtype=np.complex128))
        h = np.zeros((m.np, ld), dtype=np.complex128)
        proj = np.zeros((self.proj.nprojections, ld), dtype=np.complex128) if self.proj is not None else None
        c = self._ctx(ld, nst)
        lib().orc_hpsi(C.byref(c), _p(x.view(np.float64)), _p(h.view(np.float64)),
                       _p(proj.view(np.float64)) if proj is not None else None)
        return h[:, :nst]

    def taylor(self, psi: np.ndarray, dt, order: int = 4) -> np.ndarray:
        """exp(-i dt H) psi by the order-``order`` Taylor series; (np_part,nst) in,
        (np, nst) out."""
        m = self.mesh
        nst = psi.shape[1]
        x, ld = self.packed(np.asarray(psi, dtype=np.complex128))
        t1 = np.zeros((m.np_part, ld), dtype=np.complex128)
        t2 = np.zeros((m.np_part, ld), dtype=np.complex128)
        proj = np.zeros((self.proj.nprojections, ld), dtype=np.complex128) if self.proj is not None else None
        c = self._ctx(ld, nst)
        dt = complex(dt)
        lib().orc_taylor(C.byref(c), _p(x.view(np.float64)), C.c_double(dt.real), C.c_double(dt.imag),
                         C.c_int(order), _p(t1.view(np.float64)), _p(t2.view(np.float64)),
                         _p(proj.view(np.float64)) if proj is not None else None)
        return x[: m.np, :nst].copy()


# ---------------------------------------------------------------------------
# time propagation (exponential midpoint, td_run / exponential_midpoint)
def laser_field(E0, omega, T, t):
    """E0 sin^2(pi t/T) cos(omega t) on [0, T], zero outside."""
    if t < 0 or t > T or T <= 0:
        return 0.0
    return E0 * np.sin(np.pi * t / T) ** 2 * np.cos(omega * t)


def td_propagate(H, v0, psi, nsteps, dt, E0, omega, T, pol=(0.0, 0.0, 1.0), order=4, t0=0.0,
                 propagator="exp_mid"):
    """Exponential-midpoint propagation with the laser folded into v
    (src/td/propagator_expmid.F90:52-100, src/hamiltonian/hamiltonian_elec.F90:1028),
    or, with propagator="etrs", the independent-particle ETRS step
    exp(-i dt/2 H(t_n+1)) exp(-i dt/2 H(t_n)) (src/td/propagator_etrs.F90:70-152).

    Returns (psi_final (np, nst), energy[n], dipole[n], norm2[n]) where the
    observables are those of psi(t_n) under H(t_n), summed over the states."""
    m = H.mesh
    r = m.x[: m.np] @ np.asarray(pol, dtype=np.float64)
    x = np.array(psi, dtype=np.complex128, copy=True)
    E, D, N = [], [], []
    dv = m.vol_pp
    for n in range(nsteps):
        tn = t0 + n * dt
        H.v[:] = v0 + laser_field(E0, omega, T, tn) * r
        h = H.apply(x)
        a = x[: m.np]
        E.append(dv * float(np.sum(np.real(a.conj() * h))))
        D.append(dv * float(np.sum(np.abs(a) ** 2 * r[:, None])))
        N.append(dv * float(np.sum(np.abs(a) ** 2)))
        if propagator == "etrs":
            y = H.taylor(x, 0.5 * dt, order=order)  # H(t_n) is in place
            x = np.zeros_like(x)
            x[: m.np] = y
            H.v[:] = v0 + laser_field(E0, omega, T, tn + dt) * r
            y = H.taylor(x, 0.5 * dt, order=order)
        else:
            H.v[:] = v0 + laser_field(E0, omega, T, tn + 0.5 * dt) * r
            y = H.taylor(x, dt, order=order)
        x = np.zeros_like(x)
        x[: m.np] = y
    H.v[:] = v0
    return x[: m.np], np.array(E), np.array(D), np.array(N)


def lanczos(H, psi, dt, max_order=30, tol=1e-5):
    """exp(-i dt H) psi by the Lanczos method of exponential_lanczos_batch
    (src/electrons/exponential.F90:766-901): Krylov vectors orthogonalised by
    classical Gram-Schmidt against the last two (X(mesh_batch_orthogonalization),
    src/grid/mesh_batch_inc.F90:1168-1274), exp of the projected Hermitian matrix
    by eigendecomposition (zlalg_exp), stop when every error estimate
    |h(m+1,m) expo(m,1)| < tol after more than 3 iterations or on breakdown.
    Returns (psi_new (np, nst), dimension used, largest error estimate)."""
    m = H.mesh
    dv = m.vol_pp
    eps = np.finfo(np.float64).eps
    x = np.array(np.asarray(psi)[: m.np], dtype=np.complex128)
    nst = x.shape[1]
    beta = np.sqrt(dv * np.sum(np.abs(x) ** 2, axis=0))
    if np.all(np.abs(beta) <= 1e-12):
        return x, 0, 0.0
    V = [x / np.where(beta > 0, beta, 1.0)]
    K = max_order
    Hm = np.zeros((nst, K + 1, K + 1), dtype=np.complex128)
    expo, res, it = None, np.zeros(nst), 1
    for it in range(1, K + 1):
        pad = np.zeros((m.np_part, nst), dtype=np.complex128)
        pad[: m.np] = V[it - 1]
        w = H.apply(pad)
        lo = max(1, it - 1)
        ov = [dv * np.sum(V[j - 1].conj() * w, axis=0) for j in range(lo, it + 1)]
        for j, o in zip(range(lo, it + 1), ov):
            Hm[:, j - 1, it - 1] = o
        for j, o in zip(range(lo, it + 1), ov):
            w = w - o[None, :] * V[j - 1]
        nrm = np.sqrt(dv * np.sum(np.abs(w) ** 2, axis=0))
        Hm[:, it, it - 1] = nrm
        expo = []
        for i in range(nst):
            lam, Q = np.linalg.eigh(Hm[i, :it, :it], UPLO="U")
            expo.append((Q * np.exp(-1j * dt * lam)[None, :]) @ Q.conj().T)
        res = np.abs(nrm) * np.array([abs(e[it - 1, 0]) for e in expo])
        if np.all(np.abs(nrm) < 1e4 * eps):
            break
        w = w / np.where(np.abs(nrm) >= 1e4 * eps, np.abs(nrm), 1.0)[None, :]
        V.append(w)
        if it > 3 and np.all(res < tol):
            break
    mdim = min(it, K)
    out = np.zeros_like(x)
    for j in range(mdim):
        out += (beta * np.array([e[j, 0] for e in expo]))[None, :] * V[j]
    return out, mdim, float(np.max(res))


# ---------------------------------------------------------------------------
# dense FP64 pieces
def ghost_exchange(domains, batches):
    """Ghost rows of every partition from the owners' inner rows, in place:
    X(ghost_update_batch_start/finish) (src/grid/boundaries_inc.F90:57-231)
    with the send map packed as the ghost_reorder kernel does and each message
    landing at np_local + ghost_rdispls(source).  ``batches[p]`` is partition
    p's local (npts, ld) array."""
    for p, dp in enumerate(domains):
        for q, dq in enumerate(domains):
            n = int(dp.ghost_rcounts[q])
            if q == p or n == 0:
                continue
            so = int(dq.ghost_sdispls[p])
            rows = dq.ghost_sendmap[so: so + n]
            ro = dp.np_local + int(dp.ghost_rdispls[q])
            batches[p][ro: ro + n] = batches[q][rows]
    return batches


def kb_bra(maps, mats, scals, psi, phases=None):
    """KB projections of a batch, proj[r, s] = scal[r] * sum_k P[k, r] *
    psi[map[k], s], matrices in order: the gather and GEMM of
    X(hamiltonian_elec_base_nlocal_start)
    (src/hamiltonian/hamiltonian_elec_base_inc.F90:650-780), before the
    reduction over domains (:836)."""
    x = np.asarray(psi)
    phases = [None] * len(maps) if phases is None else phases
    # with projector phases (k != 0) the gathered points are psi(map) * phase
    # (hamiltonian_elec_base_inc.F90:680-701)
    rows = [np.asarray(sc, dtype=np.float64)[:, None] *
            (np.asarray(mt, dtype=np.float64).T @ (x[np.asarray(mp)] if ph is None else
                                                   x[np.asarray(mp)] * np.asarray(ph)[:, None]))
            for mp, mt, sc, ph in zip(maps, mats, scals, phases)]
    return np.concatenate(rows) if rows else np.zeros((0,) + x.shape[1:], dtype=x.dtype)


def kb_ket(maps, mats, proj, h, phases=None):
    """h[map[k], s] += sum_r P[k, r] * proj[r, s], in place: the GEMM and
    scatter-add of X(hamiltonian_elec_base_nlocal_finish)
    (src/hamiltonian/hamiltonian_elec_base_inc.F90:909-1027)."""
    r = 0
    phases = [None] * len(maps) if phases is None else phases
    for mp, mt, ph in zip(maps, mats, phases):
        mt = np.asarray(mt, dtype=np.float64)
        n = mt.shape[1]
        c = mt @ proj[r: r + n]
        if ph is not None:  # conjugate phase on the way back (:934-1025)
            c = c * np.conj(np.asarray(ph))[:, None]
        np.add.at(h, np.asarray(mp), c)
        r += n
    return h


def mesh_batch_nrm2(mesh, psi):
    a = np.asarray(psi)[: mesh.np]
    return np.sqrt(mesh.vol_pp * np.sum(np.abs(a) ** 2, axis=0))


def density_accumulate(mesh, psi, weight, rho=None):
    """rho + sum_i weight_i |psi_i|^2 on the inner points: the packed,
    unpolarised branch of density_calc_accumulate
    (src/states/density.F90:337-357, weights from :295-298)."""
    a = np.asarray(psi)[: mesh.np]
    w = np.asarray(weight, dtype=np.float64)
    d = (np.abs(a) ** 2) @ w
    return d if rho is None else np.asarray(rho) + d


def mesh_batch_dotp_matrix(mesh, a, b):
    a = np.asarray(a)[: mesh.np]
    b = np.asarray(b)[: mesh.np]
    return mesh.vol_pp * (a.conj().T @ b)


def cholesky_orthonormalize(mesh, psi):
    """psi (npts, nst) -> psi U^-1 with S = U^H U (upper Cholesky factor)."""
    S = mesh_batch_dotp_matrix(mesh, psi, psi)
    L = np.linalg.cholesky(S)          # S = L L^H, U = L^H
    U = L.conj().T
    out = np.linalg.solve(U.T, np.asarray(psi).T).T   # psi U^-1
    return out


def derivatives_test_error(mesh, weights, points, complex_case: bool, use_ref=True):
    """Laplacian error norm of ``X(derivatives_test)`` on ``mesh``.

    f = b exp(-a r^2) + c on all np_part points (boundaries not reset),
    res = 2 * (1/2 lapl f) - exact, printed as mf_nrm2(res)."""
    x = mesh.x
    r2 = np.sum(x ** 2, axis=1)
    a = 1.0 / float(np.max(np.abs(x[: mesh.np])) if mesh.extra.get("bbox_l") is None else mesh.extra["bbox_l"])
    a = 1.0 / mesh.extra["bbox_l"] if "bbox_l" in mesh.extra else a
    b = 10.0
    c = 100.0
    if complex_case:
        a = a + 0.01j
        b = b * np.exp(0.345j)
        c = c - 50.0j
    f = b * np.exp(-a * r2) + c
    op = Operator(mesh, points)
    w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64) * 0.5)
    fi = np.zeros((mesh.np_part, 1), dtype=np.complex128)
    fi[:, 0] = f
    fo = np.zeros((mesh.np, 1), dtype=np.complex128)
    fn = ref_operate() if use_ref else None
    fn = fn or lib().orc_operate_ri
    fn(C.byref(C.c_int(op.W)), _p(w), C.byref(C.c_int(op.nri)), _p(op.ri, C.c_int), _p(op.imin, C.c_int),
       _p(op.imax, C.c_int), _p(fi.view(np.float64)), C.byref(C.c_int(1)), _p(fo.view(np.float64)))
    res = fo[:, 0]
    if not complex_case:
        res = res.real.astype(np.complex128)  # the real build never sees imaginary parts
        f_r = (b * np.exp(-a * r2) + c)
        assert np.allclose(f_r.imag, 0)
    xi = x[: mesh.np]
    r2i = r2[: mesh.np]
    exact = 4 * a ** 2 * b * r2i * np.exp(-a * r2i) - 3 * 2 * a * b * np.exp(-a * r2i)
    res = 2 * res - exact
    return float(np.sqrt(np.sum(np.abs(res) ** 2)) * np.sqrt(mesh.vol_pp))
