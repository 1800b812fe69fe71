"""B200 Hamiltonian-apply and Taylor-propagation library (host side).

``hpsi.lib`` binds the C ABI of ``libhpsi.so``; ``hpsi.mesh``, ``hpsi.stencil``
and ``hpsi.fixtures`` are the host-side set-up a caller performs (mesh point
lists, finite-difference weights, synthetic systems).
"""
from . import mesh, stencil  # noqa: F401
