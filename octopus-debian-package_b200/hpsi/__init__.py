"""B200 Hamiltonian-apply and Taylor-propagation library (host side).

``hpsi.lib`` binds the C ABI of ``libhpsi.so``; ``hpsi.mesh``, ``hpsi.stencil``
and ``hpsi.fixtures`` are the host-side set-up a caller performs (mesh point
lists, finite-difference weights, synthetic systems); ``hpsi.obf`` reads and
writes the reference's binary restart files; ``hpsi.domain`` and
``hpsi.states_parallel`` are the multi-rank layers (domain partitions with
ghost rows, state blocks).
"""
from . import mesh, stencil  # noqa: F401
