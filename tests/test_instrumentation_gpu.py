"""The engine's tuning and instrumentation entry points through the C ABI.

* lare_gpu_set_block (the point kernels' block shape, chosen per grid size
  by the ensemble autotuner): every accepted shape gives the exact engine's
  state bit for bit (it changes only how points map to threads), and shapes
  that are not whole warps or exceed 256 threads are refused.
* lare_gpu_profile / lare_gpu_profile_report / lare_gpu_launch_count: a
  profiled step equals an unprofiled one bit for bit (the profiler only
  records events), every launch site of the step is listed with its
  launches, time and algorithmic bytes, and the launch counter advances.
* lare_gpu_field_device: the device address and strides it reports address
  the same values that lare_gpu_get_field returns.
"""
import numpy as np
import pytest

from conftest import STATE
from lare3d_b200 import decks
from lare3d_b200.abi import LareError

pytestmark = pytest.mark.gpu


def _ragged_deck():
    from test_parity_gpu import _ragged_resistive_deck
    return _ragged_resistive_deck(45, 38, 67, 5)


def _run(d, steps=3, block=None, profile=False):
    from lare3d_b200 import ensemble, gpu
    g = gpu.simulation(d, precision=gpu.EXACT64)
    if block is not None:
        ensemble.set_block(g, *block)
    g.start(d.state)
    if profile:
        g.profile(True)
    for s in range(1, steps + 1):
        g.step(s)
    return g


def test_block_shapes_give_identical_states(built):
    d = _ragged_deck()
    ref = _run(d)
    want = {f: ref.get_field(f) for f in STATE}
    ref.close()
    for block in ((64, 2), (32, 8), (128, 1), (256, 1), (32, 2)):
        g = _run(_ragged_deck(), block=block)
        for f in STATE:
            assert np.array_equal(g.get_field(f), want[f]), (block, f)
        g.close()


def test_block_shape_checks(built):
    from lare3d_b200 import ensemble, gpu
    d = decks.blast(12)
    g = gpu.simulation(d, precision=gpu.FP64)
    for bad in ((33, 1), (0, 4), (32, 16), (16, 1)):
        with pytest.raises(LareError):
            ensemble.set_block(g, *bad)
    ensemble.set_block(g, 64, 4)
    g.close()


def test_profiled_step_is_unchanged_and_reported(built):
    d = _ragged_deck()
    plain = _run(d, steps=2)
    want = {f: plain.get_field(f) for f in STATE}
    plain.close()
    g = _run(_ragged_deck(), steps=1, profile=True)
    before = g.launch_count()
    g.step(2)
    assert g.launch_count() > before + 30  # a resistive MHD step is several dozen launches
    for f in STATE:
        assert np.array_equal(g.get_field(f), want[f]), f
    rep = g.profile_report()
    sites = {p["site"] for p in rep}
    for s in ("remap_sweep_bupd", "remap_sweep_bflux_march", "remap_sweep_bflux_x", "shock_heating",
              "shock_viscosity_lp4_tile", "set_dt_min", "corrector_visc_heating_sum", "ohmic_heating_sum",
              "eta_and_rkstep", "ghost"):
        assert any(x.split(":")[0] == s for x in sites), (s, sorted(sites))
    for p in rep:
        assert p["launches"] >= 1 and p["ms"] > 0.0, p
        assert p["bytes"] >= 0.0 and (p["words"] == 0) == (p["bytes"] == 0.0), p
    g.close()


@pytest.mark.parametrize("precision", [64, 32])
def test_field_device_addresses_the_fields(built, precision):
    import torch
    from lare3d_b200 import gpu
    d = decks.orszag_tang(12)
    g = gpu.simulation(d, precision=precision)
    g.start(d.state)
    g.step(1)
    torch.cuda.synchronize()
    for name in ("rho", "energy", "vx", "bz"):
        origin, sx, sxy, eb = g.field_device(name)
        assert origin != 0 and eb == (8 if precision == 64 else 4)
        assert sx >= d.nx + 5 and sx % 4 == 0 and sxy == sx * (d.ny + 5)
        host = g.get_field(name)
        lo, _ = g.field_bounds(name)
        # the whole padded allocation starts at Fortran (-2, -2, -2)
        n = sxy * (d.nz + 5)
        first = origin - (2 + 2 * sx + 2 * sxy) * eb

        class View:  # a zero-copy view of the allocation (CUDA array interface)
            __cuda_array_interface__ = {"shape": (n,), "typestr": "<f8" if eb == 8 else "<f4",
                                        "data": (first, False), "version": 2}

        dev = torch.as_tensor(View(), device="cuda").double().cpu().numpy()
        for (i, j, k) in ((0, 0, 0), (1, 2, 3), (d.nx, d.ny, d.nz), (-1, 0, 2)):
            want = host[i - lo[0], j - lo[1], k - lo[2]]
            got = dev[(i + 2) + sx * (j + 2) + sxy * (k + 2)]
            assert got == want, (name, i, j, k, got, want)
    g.close()
