"""Allocation-free norm entry point (collected last on purpose).

hpsi_nrm2_noalloc serves callers that must not let the library allocate
device memory (an application that owns the device-memory budget, or a
per-step loop that may not reach the allocator).  It keeps its partial sums
in a fixed device array of the library instead of a mesh workspace.  This
test calls it through the C ABI twice in a row and compares each result with
the allocating hpsi_nrm2 at the reduction tolerance the other tests use.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13


def test_nrm2_noalloc_matches_nrm2(cuda):
    import torch
    from hpsi import fixtures, lib
    from hpsi.mesh import sphere_mesh

    rng = np.random.default_rng(41)
    m = sphere_mesh(3.0, 0.3)
    psi = fixtures.random_states(m, 6, rng, orthonormal=False)
    for dtype in (np.complex128, np.complex64):
        x = torch.from_numpy(np.ascontiguousarray(psi.astype(dtype))).to(cuda)
        dm = lib.DeviceMesh(m)
        ref = dm.nrm2(x)
        for _ in range(2):
            got = lib.nrm2_noalloc(m.np, m.vol_pp, x)
            assert np.max(np.abs(got - ref) / ref) <= TOL
        # device output, read back after the stream finishes
        dout = torch.zeros(6, dtype=torch.float64, device=cuda)
        b = lib.as_batch(x)
        lib.check(lib.load().hpsi_nrm2_noalloc(m.np, m.vol_pp, C.byref(b),
                                               C.cast(dout.data_ptr(), C.POINTER(C.c_double)),
                                               lib._stream_ptr(None)))
        torch.cuda.synchronize()
        assert np.max(np.abs(dout.cpu().numpy() - ref) / ref) <= TOL
        dm.close()


def test_nrm2_noalloc_rejects_too_many_states(cuda):
    import torch
    from hpsi import lib
    x = torch.zeros((10, 512), dtype=torch.complex128, device=cuda)
    with pytest.raises(lib.HpsiError) as e:
        lib.nrm2_noalloc(10, 1.0, x)
    assert e.value.status == 1
    assert "exceed the maximum" in str(e.value)
