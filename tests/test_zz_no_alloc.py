"""GPU test of lare_gpu_energy_noalloc, the allocation-free energy budget.

That entry point serves callers that keep the state in their own device
memory and cannot let the library call cudaMalloc (a fixed device pool, or
no allocation between stream-ordered steps).  It must return what the
context-based lare_gpu_energy returns for the same state, within the energy
tolerance the other tests use (relative 1e-12), on consecutive calls that
share its fixed scratch.  This file is collected last so that a run stopping
at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATE = ["rho", "energy", "vx", "vy", "vz", "bx", "by", "bz"]


def entry():
    from lare3d_b200 import gpu
    fn = gpu.library().lare_gpu_energy_noalloc
    fn.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 13
    fn.restype = C.c_int
    return fn


def test_energy_noalloc_matches_context_energy(built):
    import torch
    from lare3d_b200 import decks, gpu
    fn = entry()
    n = 16
    d = decks.orszag_tang(n)
    sim = gpu.simulation(d)
    sim.start(d.state)
    mets = [torch.from_numpy(np.ascontiguousarray(d.metrics[k])).cuda() for k in ("dxb", "dyb", "dzb")]
    stream = torch.cuda.current_stream().cuda_stream
    results = []
    for call in range(2):
        # a different state for each call, so the second call cannot pass on
        # scratch contents left by the first
        sim.step(call + 1)
        ref = sim.energy()[:3]
        st = sim.download()
        dev = [torch.from_numpy(st[k].ravel(order="F").copy()).cuda() for k in STATE]
        out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
        rc = fn(n, n, n, *[t.data_ptr() for t in dev], *[t.data_ptr() for t in mets], out.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        for q in range(3):
            assert abs(got[q] - ref[q]) <= 1e-12 * abs(ref[q]), (call, q, got[q], ref[q])
        results.append(got)
    assert not np.array_equal(results[0], results[1])
    sim.close()


def test_energy_noalloc_rejects_oversize_grid(built):
    fn = entry()
    # 400^3 exceeds LARE_NOALLOC_MAX_POINTS; rejected before any pointer is used
    assert fn(400, 400, 400, *([None] * 12), None) == -8
    assert fn(0, 8, 8, *([None] * 12), None) == -1
