"""State-parallel propagation on the CPU: the reference's block division
rule, and the observable sum over two gloo ranks (the per-block propagation
stands in for the device call with the oracle's H psi)."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import small_sphere_system

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("nobjs,nprocs,want", [
    (10, 3, [(0, 4), (4, 7), (7, 10)]),
    (12, 4, [(0, 3), (3, 6), (6, 9), (9, 12)]),
    (7, 1, [(0, 7)]),
    (2, 4, [(0, 1), (1, 2), (2, 2), (2, 2)]),
    (0, 2, [(0, 0), (0, 0)]),
])
def test_divide_range_cases(nobjs, nprocs, want):
    from hpsi.states_parallel import divide_range
    assert divide_range(nobjs, nprocs) == want


def test_divide_range_covers_every_object_once():
    from hpsi.states_parallel import divide_range
    for nobjs in range(0, 40):
        for nprocs in range(1, 12):
            r = divide_range(nobjs, nprocs)
            got = [i for a, b in r for i in range(a, b)]
            assert got == list(range(nobjs))
            sizes = [b - a for a, b in r]
            if nprocs <= nobjs:
                assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    with pytest.raises(ValueError):
        divide_range(3, 0)


class _OracleBlock:
    """Stand-in for the device td_propagate: per step the energy, dipole and
    norm sums of the block under the oracle's H (the states are not moved;
    the test checks the split and the sum)."""

    def __init__(self, H, m):
        self.H, self.m = H, m

    def td_propagate(self, psi, nsteps, dt):
        h = self.H.apply(psi)
        a = psi[: self.m.np]
        dv = self.m.vol_pp
        e = dv * np.sum(np.real(np.conj(a) * h))
        d = dv * np.sum(np.abs(a) ** 2 * self.m.x[: self.m.np, 2:3])
        n = dv * np.sum(np.abs(a) ** 2)
        k = np.arange(1, nsteps + 1)
        return e * k, d * k, n * k


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, nst, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "octopus-debian-package_b200"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from helpers import small_sphere_system
    from hpsi.states_parallel import divide_range, td_propagate_states
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O
    m, v, proj, psi = small_sphere_system(seed=59, nst=nst)
    H = O.Hamiltonian(m, laplacian_weights(m.spacing), star_points(), v=v,
                      projectors=O.Projectors(proj.maps, proj.mats, proj.scals))
    a, b = divide_range(nst, world)[rank]
    blk = np.ascontiguousarray(psi[:, a:b]) if b > a else None
    e, d, n = td_propagate_states(_OracleBlock(H, m), blk, 5, 0.02)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, (e, d, n)))


@pytest.mark.parametrize("nst", [5, 1])
def test_observables_summed_over_two_gloo_ranks(nst):
    from hpsi.stencil import laplacian_weights, star_points
    from oracle import oracle as O
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, nst, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    m, v, proj, psi = small_sphere_system(seed=59, nst=nst)
    H = O.Hamiltonian(m, laplacian_weights(m.spacing), star_points(), v=v,
                      projectors=O.Projectors(proj.maps, proj.mats, proj.scals))
    want = _OracleBlock(H, m).td_propagate(psi, 5, 0.02)
    for r in range(world):
        for got, ref in zip(res[r], want):
            assert np.allclose(got, ref, rtol=1e-12, atol=0)
