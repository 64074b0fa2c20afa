"""GPU parity of branches the plain workloads leave off, and of the restart
path, through the C ABI against the oracle.

* Boris correction (control.f90:183 ``boris``, ``va_max``): set_dt lowers
  gamma_boris where the Alfven speed exceeds va_max (lagran.F90:1104-1109),
  and the reduced factor enters the sound speed of shock_viscosity (:556)
  and the Lorentz force of the predictor (:375-377).
* Gravity (lagran.F90:379, ``fz = fz - rho_v*grav(iz)``) with a profile that
  varies along z.
* Conduction without the Larsen heat-flux limiter (``heat_flux_limiter`` =
  .FALSE., conduct.f90:99-110 and :236-246).
* Restart (lare3d.f90:55-59, setup.F90:518-688): a run continued from a
  downloaded state in a fresh context with ``restart`` set; the first set_dt
  takes dt_from_restart and returns before advancing the time
  (lagran.F90:1080-1086).

The exact FP64 engine must agree bit for bit (conduction, whose pow differs
in the last bit, at relative L2 1e-12); the product FP64 engine within
relative L2 1e-10.
"""
import numpy as np
import pytest

from conftest import STATE, rel_l2
from lare3d_b200 import decks
from lare3d_b200.abi import LareError

pytestmark = pytest.mark.gpu


def sims(deck, precision, grav=None):
    from lare3d_b200 import gpu
    from oracle import oracle
    r = oracle.simulation(deck)
    g = gpu.simulation(deck, precision=precision)
    r.start(deck.state, grav=grav)
    g.start(deck.state, grav=grav)
    return r, g


def check(g, r, names, exact, tag):
    for f in names:
        a, b = g.get_field(f), r.get_field(f)
        if exact:
            nbad = int(np.count_nonzero(a != b))
            assert nbad == 0, f"{tag}: {f} differs in {nbad} elements (max |d| {np.abs(a - b).max():.3e})"
        else:
            e = rel_l2(a, b)
            assert e <= 1e-10, f"{tag}: {f} rel L2 {e:.2e}"


@pytest.mark.parametrize("precision", ["exact", "product"])
def test_boris_correction(built, precision):
    from lare3d_b200 import gpu
    d = decks.orszag_tang(16, boris=1, va_max=0.3)
    exact = precision == "exact"
    r, g = sims(d, gpu.EXACT64 if exact else gpu.FP64)
    for s in range(1, 6):
        r.step(s)
        g.step(s)
        check(g, r, STATE + ["gamma_boris", "p_visc", "pressure"], exact, f"step {s}")
        assert g.scalars().dt == r.scalars().dt if exact else abs(g.scalars().dt / r.scalars().dt - 1) < 1e-12
    gb = r.get_field("gamma_boris")
    assert gb.min() < 0.6, "va_max must bind somewhere"
    # the correction changes the run: without it dt is set by the full Alfven speed
    d0 = decks.orszag_tang(16)
    r0, _ = sims(d0, gpu.EXACT64)
    r0.step(1)
    r1, _ = sims(d, gpu.EXACT64)
    r1.step(1)
    assert r1.scalars().dt > r0.scalars().dt


def _grav_profile(d):
    zc = d.metrics["zc"]                       # cell centres -1:nz+2, as grav
    return np.ascontiguousarray(0.5 * (1.0 + 0.3 * np.sin(2.0 * np.pi * zc)))


@pytest.mark.parametrize("precision", ["exact", "product"])
def test_gravity(built, precision):
    from lare3d_b200 import gpu
    d = decks.blast(16)
    grav = _grav_profile(d)
    exact = precision == "exact"
    r, g = sims(d, gpu.EXACT64 if exact else gpu.FP64, grav=grav)
    for s in range(1, 6):
        r.step(s)
        g.step(s)
        check(g, r, STATE, exact, f"step {s}")
    # gravity acts: the run differs from the same deck without it
    _, g0 = sims(d, gpu.EXACT64)
    for s in range(1, 6):
        g0.step(s)
    assert rel_l2(g0.get_field("vz"), g.get_field("vz")) > 1e-3


def test_gravity_uniform_state_falls_freely(built):
    """A uniform state in a uniform field g: no pressure or magnetic force,
    so the predictor-corrector gives every vertex vz = -g dt after one step
    (v1 = -g dt/2, v = 2 v1 - v0), which the remap of a uniform velocity
    keeps; both engines reproduce it to round-off."""
    from lare3d_b200 import gpu
    d = decks.blast(12)
    st = d.state
    st["energy"][...] = 0.1 / ((d.params.gamma - 1.0) * 1.0)
    g0 = 0.7
    grav = np.full(d.metrics["zc"].shape, g0)
    for prec in (gpu.EXACT64, gpu.FP64, gpu.FP32):
        s = gpu.simulation(d, precision=prec)
        s.start(st, grav=grav)
        s.step(1)
        dt = s.scalars().dt
        vz = s.get_field("vz")[2:-2, 2:-2, 2:-2]
        tol = 1e-5 if prec == gpu.FP32 else 1e-13
        assert np.abs(vz + g0 * dt).max() <= tol * g0 * dt, prec
        s.close()


@pytest.mark.parametrize("in_step", [False, True])
def test_conduction_without_flux_limiter(built, in_step):
    from lare3d_b200 import gpu
    if in_step:
        d = decks.conduction(12, kappa_0=1.0e-4, heat_flux_limiter=0)
    else:
        d = decks.conduction(16, heat_flux_limiter=0)
    for prec, tol in ((gpu.EXACT64, 1e-12), (gpu.FP64, 1e-10)):
        r, g = sims(d, prec)
        for it in range(1, 3):
            if in_step:
                r.step(it)
                g.step(it)
                names = STATE
            else:
                assert r.conduct_heat(d.dt_fixed) == g.conduct_heat(d.dt_fixed)
                names = ["energy", "temperature"]
            assert r.scalars().n_s_stages == g.scalars().n_s_stages
            for f in names:
                assert rel_l2(g.get_field(f), r.get_field(f)) <= tol, (prec, it, f)
    # the limiter matters on this deck: with it on, the energy differs
    dl = decks.conduction(16, heat_flux_limiter=1)
    if not in_step:
        a, _ = sims(d, gpu.EXACT64)
        b, _ = sims(dl, gpu.EXACT64)
        a.conduct_heat(d.dt_fixed)
        b.conduct_heat(d.dt_fixed)
        assert rel_l2(a.get_field("energy"), b.get_field("energy")) > 1e-8


def _restart_sequence(make_sim, d, first, total, dt_from_restart, dt_start=0.0):
    """`first` steps in one context, then a fresh context with restart set,
    the downloaded state and the saved time, stepping on to `total`.
    dt_start is the dt the driver holds before the first step (a restarted
    reference process has not set it: 0; shock_viscosity reads it before
    set_dt runs, lagran.F90:129-130)."""
    a = make_sim(d)
    a.start(d.state)
    for s in range(1, first + 1):
        a.step(s)
    saved = a.download()
    t_saved = a.scalars().time
    a.close()
    p = d.params
    old = (p.restart, p.dt_from_restart)
    p.restart, p.dt_from_restart = 1, dt_from_restart
    try:
        b = make_sim(d)
    finally:
        p.restart, p.dt_from_restart = old
    b.start(saved, time=t_saved, dt=dt_start)
    b.step(first + 1)
    sc = b.scalars()
    first_dt, first_time = sc.dt, sc.time
    for s in range(first + 2, total + 1):
        b.step(s)
    return b, t_saved, first_dt, first_time


def test_restart(built):
    from lare3d_b200 import gpu
    from oracle import oracle
    d = decks.blast(12)
    # the uninterrupted run, and the dt its step 6 takes
    ref = gpu.simulation(d, precision=gpu.EXACT64)
    ref.start(d.state)
    dts, times = {}, {}
    for s in range(1, 11):
        ref.step(s)
        dts[s], times[s] = ref.scalars().dt, ref.scalars().time
    # (1) GPU and oracle take the same restart path bit for bit, with the dt
    # a dump holds (the last step's, diagnostics.F90 writes dt)
    out = []
    for make in (lambda dk: oracle.simulation(dk), lambda dk: gpu.simulation(dk, precision=gpu.EXACT64)):
        out.append(_restart_sequence(make, d, 5, 10, dts[5]))
    (r, tr, dtr0, timer), (g, tg, dtg0, timeg) = out
    for f in STATE:
        assert np.array_equal(g.get_field(f), r.get_field(f)), f
    assert (tg, dtg0, timeg) == (tr, dtr0, timer)
    # the first set_dt after a restart takes dt_from_restart and leaves the
    # time where the dump left it (lagran.F90:1080-1086)
    assert dtg0 == dts[5] and timeg == tg
    # (2) given the dt the uninterrupted run's step 6 takes, the continued run
    # equals the uninterrupted one bit for bit (state round trip through
    # download/upload, ghosts refilled by the boundary conditions); its clock
    # lags by the one step whose dt was not added.  The driver holds the last
    # step's dt, as the uninterrupted run's shock viscosity sees it.
    g2, _, dt6, _ = _restart_sequence(lambda dk: gpu.simulation(dk, precision=gpu.EXACT64), d, 5, 10, dts[6],
                                      dt_start=dts[5])
    assert dt6 == dts[6]
    for f in STATE:
        assert np.array_equal(g2.get_field(f), ref.get_field(f)), f
    assert abs(g2.scalars().time - (times[10] - dts[6])) <= 1e-14 * times[10]


def test_restart_of_a_resistive_run_reports_dt_error(built):
    """The reference's first set_dt after a restart returns before setting
    dtr (lagran.F90:1080-1086), so a resistive restart divides by a dtr that
    was never set (lagran.F90:137-139).  The library refuses that step with
    LARE_EDT instead of sub-cycling on an undefined count."""
    from lare3d_b200 import gpu
    d = decks.orszag_tang(8)
    d.params.restart, d.params.dt_from_restart = 1, 1e-3
    g = gpu.simulation(d, precision=gpu.FP64)
    g.start(d.state)
    with pytest.raises(LareError) as e:
        g.step(1)
    assert e.value.code == -4
