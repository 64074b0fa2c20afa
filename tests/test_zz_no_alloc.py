"""GPU test of lare_gpu_energy_noalloc, the allocation-free energy budget.

That entry point serves callers that keep the state in their own device
memory and cannot let the library call cudaMalloc (a fixed device pool, or
no allocation between stream-ordered steps).  It must return what the
context-based lare_gpu_energy returns for the same state, within the energy
tolerance the other tests use (relative 1e-12), on consecutive calls that
share its fixed scratch.  Grids of one block (16^3: 4913 vertices, below the
8192 points a block sums), of several blocks (32^3: 5 blocks) and a ragged
grid (37 x 29 x 41: 6 blocks) cover the split of the cell and vertex loops
across blocks and the strided final sum.  This file is collected last so that
a run stopping at the first failure has already run every other test.
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


def _ragged_deck(nx, ny, nz, seed):
    from lare3d_b200 import decks
    from lare3d_b200.abi import State
    from lare3d_b200.grid import grid
    d = decks.orszag_tang(8)
    m = grid(nx, ny, nz, (0, 1.1), (0, 0.9), (0, 1.6))
    st = State.zeros(nx, ny, nz)
    rng = np.random.default_rng(seed)
    for k in STATE:
        lo, hi = (0.5, 1.5) if k in ("rho", "energy") else (-0.3, 0.3)
        st[k][...] = rng.uniform(lo, hi, st[k].shape)
    return decks.Deck("ragged", d.params, nx, ny, nz, m, st, nsteps=2)


def _decks():
    from lare3d_b200 import decks
    return [decks.orszag_tang(16), decks.orszag_tang(32), _ragged_deck(37, 29, 41, 5)]


@pytest.mark.parametrize("case", [0, 1, 2], ids=["16^3-one-block", "32^3-five-blocks", "37x29x41-ragged"])
def test_energy_noalloc_matches_context_energy(built, case):
    import torch
    from lare3d_b200 import gpu
    fn = entry()
    d = _decks()[case]
    nx, ny, nz = d.nx, d.ny, d.nz
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
        rc = fn(nx, ny, nz, *[t.data_ptr() for t in dev], *[t.data_ptr() for t in mets], out.data_ptr(), stream)
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
