"""GPU checks of batched ensembles: one graph launch per 6 steps of every
member gives each member exactly the state of the same run stepped alone
(FP32 form, bit for bit, resistive sub-cycles included), whatever block
shape the autotuner picked; and the host-side rules of lare_ens_create."""
import ctypes as C

import numpy as np
import pytest

from conftest import STATE

pytestmark = pytest.mark.gpu


def specs():
    from lare3d_b200.ensemble import MemberSpec
    return [MemberSpec("blast", 16, 0.5, 1e-3, 3), MemberSpec("orszag_tang", 24, 0.05, 5e-3, 4),
            MemberSpec("blast", 20, 5.0, 1e-4, 5), MemberSpec("orszag_tang", 16, 2.0, 1e-2, 6)]


def test_ensemble_matches_single_runs(built):
    from lare3d_b200 import gpu
    from lare3d_b200.ensemble import Ensemble, member_deck
    ds = [member_deck(s) for s in specs()]
    ens = Ensemble(ds, precision=32, blocks={16: (32, 4), 24: (128, 2), 20: (32, 8)})
    ens.launch(2)
    ens.sync()
    assert ens.steps == 13
    for i, d in enumerate(ds):
        ref = gpu.simulation(d, precision=32)
        ref.start(d.state)
        for s in range(1, 14):
            ref.step(s)
        got = ens.sims[i]
        for f in STATE:
            a, b = got.get_field(f), ref.get_field(f)
            assert np.array_equal(a, b), (i, f, float(np.abs(a - b).max()))
        sa, sb = got.scalars(), ref.scalars()
        assert sa.time == sb.time and sa.dt == sb.dt and sa.steps_taken == sb.steps_taken == 13
        ref.close()
    ens.close()


def test_ensemble_create_rules(built):
    from lare3d_b200 import decks, gpu
    from lare3d_b200.ensemble import _lib
    lib = _lib()
    d = decks.blast(12)
    a = gpu.simulation(d, precision=32)
    a.start(d.state)
    h = C.c_void_p()
    arr = (C.c_void_p * 1)(a.ctx.value)
    assert lib.lare_ens_create(arr, 1, 6, C.byref(h)) == -1          # no eager step yet
    a.step(1)
    assert lib.lare_ens_create(arr, 1, 5, C.byref(h)) == -1          # not a multiple of 6
    two = (C.c_void_p * 2)(a.ctx.value, a.ctx.value)
    assert lib.lare_ens_create(two, 2, 6, C.byref(h)) == -1          # the same member twice
    c = decks.conduction(16)
    b = gpu.simulation(c, precision=32)
    b.start(c.state)
    b.step(1)
    arr = (C.c_void_p * 1)(b.ctx.value)
    assert lib.lare_ens_create(arr, 1, 6, C.byref(h)) == -1          # conduction needs the host
    arr = (C.c_void_p * 1)(a.ctx.value)
    assert lib.lare_ens_create(arr, 1, 6, C.byref(h)) == 0
    assert lib.lare_ens_launch(h, 1) == 0
    bad = C.c_int(7)
    assert lib.lare_ens_sync(h, C.byref(bad)) == 0 and bad.value == -1
    lib.lare_ens_destroy(h)
    assert a.scalars().steps_taken == 7
    a.close()
    b.close()


def test_autotune_picks_a_measured_shape(built):
    from lare3d_b200.ensemble import BLOCKS, autotune
    best, times = autotune(16, blocks=BLOCKS[:3], launches=1, kind="blast")
    assert best in BLOCKS[:3] and set(times) == set(BLOCKS[:3])
    assert all(t > 0 for t in times.values())


def test_ensemble_with_the_widened_physics(built):
    """Recorded steps carry the partially ionised models (neutral_fraction at
    each step start and in the device-side sub-cycle loop), radiation and
    rke's energy_correction: FP64 members match their single runs bit for
    bit."""
    from lare3d_b200 import decks, gpu
    from lare3d_b200.ensemble import Ensemble
    ds = [decks.partially_ionised(12, eta_bar=1e-2), decks.radiative_blast(12),
          decks.orszag_tang(12, rke=1), decks.partially_ionised(10, cowling=False, rke=1),
          decks.open_blast(12, cooling_term=1), decks.orszag_tang(10, coronal_heating=1, cooling_term=1)]
    heat = np.asfortranarray(np.full(ds[5].state["rho"].shape, 1e-3))
    ens = Ensemble(ds, precision=64, fields={5: {"heat_in": heat}})
    ens.launch(1)
    ens.sync()
    for i, d in enumerate(ds):
        ref = gpu.simulation(d, precision=64)
        ref.start(d.state)
        if i == 5:
            ref.set_field("heat_in", heat)
        for s in range(1, 8):
            ref.step(s)
        got = ens.sims[i]
        for f in STATE:
            a, b = got.get_field(f), ref.get_field(f)
            assert np.array_equal(a, b), (i, f, float(np.abs(a - b).max()))
        ref.close()
    ens.close()


def test_snapshot_pairs_match_single_run_pairs(built):
    """Training pairs from ensemble members (ensemble.snapshot_pairs): the
    member state after a graph launch, loaded into a conduction context and
    advanced by one plain RKL2 step, gives the same features and dT, bit for
    bit, as the same deck stepped alone through lare_gpu_step and turned
    into a pair by hand."""
    import torch
    from lare3d_b200 import decks, gpu
    from lare3d_b200 import surrogate as S
    from lare3d_b200.ensemble import Ensemble, member_deck, snapshot_pairs
    ds = [member_deck(s) for s in specs()[:2]]
    ens = Ensemble(ds, precision=32)
    ens.launch(1)
    ens.sync()
    pairs = snapshot_pairs(ens, [0, 1])
    meta = {"t_scale": 0.1, "rho_scale": 1.0}
    for i, d in enumerate(ds):
        ref = gpu.simulation(d, precision=32)
        ref.start(d.state)
        for s in range(1, ens.steps + 1):
            ref.step(s)
        st = ref.download()
        ref.close()
        p = decks.default_params(gamma=d.params.gamma, conduction=1, heat_flux_limiter=1, flux_limiter=0.1,
                                 kappa_0=1.0e-3, dt_multiplier=0.9)
        cd = decks.Deck("pair", p, d.nx, d.ny, d.nz, d.metrics, st, nsteps=1)
        dt = 50.0 * decks.dt_parab_estimate(st, d.metrics, p, d.nx)
        sim = gpu.simulation(cd, precision=32)
        sim.start(st)
        n = d.nx
        feat = torch.empty((5, n, n, n), dtype=torch.float32, device="cuda")
        dT = torch.empty((n, n, n), dtype=torch.float32, device="cuda")
        S.extract(sim, feat, dT, 0, meta)
        sim.conduct_heat(dt)
        S.extract(sim, None, dT, 1, meta)
        torch.cuda.synchronize()
        sim.close()
        assert torch.equal(pairs[i][0], feat), i
        assert torch.equal(pairs[i][1], dT), i
        assert float(dT.abs().max()) > 0.0, "the conduction step moves heat"
    ens.close()
