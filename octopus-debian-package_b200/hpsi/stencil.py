"""Finite-difference star stencil and its Laplacian weights (host-side setup).

The Fortran host owns the derivatives set-up and hands the library a solved
weight array; this module is the Python host's equivalent of that set-up, so
that the library, the oracle and the tests all consume the *same* FP64 array.

Reference behaviour restated here:

* ``stencil_star_get_lapl`` (src/grid/stencil_star.F90:59-93): the star points
  are ordered axis by axis, ``-order..order`` along x (the centre is taken only
  once, on the x axis), then ``-order..-1, 1..order`` along y and along z.
* ``stencil_star_polynomials_lapl`` (src/grid/stencil_star.F90:97-116): the
  polynomial basis is the constant followed by x^1..x^(2*order), then the same
  powers of y and of z.
* ``derivatives_make_discretization`` (src/grid/derivatives.F90:639-757) builds
  ``mat(j, i) = prod_k x_k(i)**pol(k, j)`` with ``x = point * spacing`` and
  ``get_rhs_lapl`` (src/grid/derivatives.F90:586-609) sets ``rhs = 2`` on the
  x^2, y^2, z^2 rows.  The system is solved with LAPACK ``dgesvx`` (no
  equilibration, iterative refinement) as in ``dlinsyssolve``
  (src/math/lalg_adv_lapack_inc.F90:806-879).
"""
from __future__ import annotations

import numpy as np


def star_points(order: int = 4, dim: int = 3) -> np.ndarray:
    """Stencil offsets, shape (W, 3), in the reference's point order."""
    pts = []
    got_center = False
    for axis in range(dim):
        for j in range(-order, order + 1):
            if j == 0:
                if got_center:
                    continue
                got_center = True
            p = [0, 0, 0]
            p[axis] = j
            pts.append(p)
    return np.asarray(pts, dtype=np.int32)


def center_index(points: np.ndarray) -> int:
    """Index of the (0,0,0) point (``stencil_init_center``)."""
    return int(np.nonzero(np.all(points == 0, axis=1))[0][0])


def star_polynomials(order: int = 4, dim: int = 3) -> np.ndarray:
    """Polynomial exponents, shape (npoly, 3)."""
    pol = [[0, 0, 0]]
    for axis in range(dim):
        for j in range(1, 2 * order + 1):
            p = [0, 0, 0]
            p[axis] = j
            pol.append(p)
    return np.asarray(pol, dtype=np.int64)


def laplacian_weights(spacing, order: int = 4) -> np.ndarray:
    """Solve for the FP64 Laplacian weights of the order-``order`` star stencil.

    Returns an array of W = 6*order+1 weights in :func:`star_points` order.
    """
    h = np.broadcast_to(np.asarray(spacing, dtype=np.float64), (3,))
    pts = star_points(order)
    pol = star_polynomials(order)
    W = len(pts)
    x = pts.astype(np.float64) * h[None, :]
    mat = np.empty((len(pol), W), dtype=np.float64)
    mat[0, :] = 1.0
    pow_max = int(pol.max())
    for i in range(W):
        powers = np.zeros((3, pow_max + 1))
        powers[:, 0] = 1.0
        for j in range(3):
            powers[j, 1] = x[i, j]
            for k in range(2, pow_max + 1):
                powers[j, k] = x[i, j] * powers[j, k - 1]
        for j in range(1, len(pol)):
            v = powers[0, pol[j, 0]]
            for k in range(1, 3):
                v = v * powers[k, pol[j, k]]
            mat[j, i] = v
    rhs = np.zeros((len(pol), 1))
    for j in range(len(pol)):
        for i in range(3):
            if pol[j, i] == 2 and all(pol[j, k] == 0 for k in range(3) if k != i):
                rhs[j, 0] = 2.0
    try:
        from scipy.linalg import lapack
        res = lapack.dgesvx(mat, rhs, fact="N", trans="N")
        sol = res[7] if isinstance(res, tuple) else res
        info = res[-1]
        if info != 0 and info != W + 1:
            raise RuntimeError(f"dgesvx info={info}")
        sol = np.asarray(sol).reshape(W)
    except ImportError:  # pragma: no cover - scipy is part of the image
        sol = np.linalg.solve(mat, rhs).reshape(W)
    return np.ascontiguousarray(sol, dtype=np.float64)
