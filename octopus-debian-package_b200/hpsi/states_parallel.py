"""State-parallel propagation: the states split into contiguous blocks, one
block per rank, each rank propagating its block on its own GPU.

With a frozen potential no term of H psi or of the Taylor step couples two
states, so the blocks need no exchange while they propagate; the per-step
observables (energy, dipole, norm: sums over states) are summed over the
ranks with one FP64 all-reduce of 3 * nsteps doubles after the propagation
(the reference sums them over st%mpi_grp as it writes them, td_write).

``divide_range`` is the reference's rule for the block of each rank,
multicomm_divide_range without ScaLAPACK (src/basic/multicomm.F90:960-1032),
which states_elec_distribute_nodes (src/states/states_elec.F90:1762-1834)
applies to the states through distributed_init
(src/basic/distributed.F90:116).
"""
from __future__ import annotations

import numpy as np


def divide_range(nobjs: int, nprocs: int) -> list[tuple[int, int]]:
    """0-based half-open [start, stop) of each rank: contiguous blocks, the
    first nobjs % nprocs ranks one longer; with more ranks than objects,
    rank i < nobjs gets object i and the others none."""
    if nprocs < 1 or nobjs < 0:
        raise ValueError("divide_range: need nprocs >= 1 and nobjs >= 0")
    if nprocs > nobjs:
        return [(i, i + 1) if i < nobjs else (nobjs, nobjs) for i in range(nprocs)]
    base, extra = divmod(nobjs, nprocs)
    out = []
    for r in range(nprocs):
        if r < extra:
            start = r * (base + 1)
            out.append((start, start + base + 1))
        else:
            stop = nobjs - (nprocs - r - 1) * base
            out.append((stop - base, stop))
    return out


def td_propagate_states(ham, psi_block, nsteps: int, dt: float, group=None, **kwargs):
    """Propagate this rank's block (``ham.td_propagate``; ``psi_block`` None
    for a rank without states) and return the per-step (energy, dipole,
    norm2) summed over the ranks of ``group``.  Every rank calls it with the
    same ``nsteps``; the one collective comes after the propagation."""
    import torch
    import torch.distributed as dist
    if psi_block is not None:
        e, d, n = ham.td_propagate(psi_block, nsteps, dt, **kwargs)
    else:
        e = d = n = np.zeros(nsteps)
    obs = np.stack([np.asarray(e, dtype=np.float64), np.asarray(d, dtype=np.float64),
                    np.asarray(n, dtype=np.float64)])
    if dist.is_available() and dist.is_initialized():
        dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        t = torch.from_numpy(obs).to(dev)
        dist.all_reduce(t, group=group)
        obs = t.cpu().numpy()
    return obs[0], obs[1], obs[2]
