"""The partially ionised plasma on the oracle (neutral.f90): its exponential,
the neutral fraction's bisection, the Cowling resistivity against a numpy
restatement, and properties of whole steps (mass conservation, the error a
cell with no temperature bracket raises, the Cowling terms' extra heating)."""
import ctypes as C

import numpy as np
import pytest

from conftest import STATE
from lare3d_b200 import decks
from lare3d_b200.abi import EOS_ION, EOS_PI, LareError


def _sim(d):
    from oracle import oracle
    s = oracle.simulation(d)
    s.start(d.state)
    return s


def test_exponential_within_one_ulp_of_numpy():
    from oracle import oracle
    f = oracle.library().lare_ref_exp
    f.argtypes = [C.c_double]
    f.restype = C.c_double
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.uniform(-745.0, 709.7, 20000), rng.uniform(-3.0, 3.0, 20000),
                        rng.uniform(-1e-6, 1e-6, 2000), np.array([0.0, -0.0, 1.0, -1.0, 709.78, -745.13])])
    got = np.array([f(float(v)) for v in x])
    want = np.exp(x)
    normal = want > np.finfo(np.float64).tiny
    ulp = np.abs(got[normal] - want[normal]) / np.spacing(want[normal])
    assert ulp.max() <= 1.0
    assert np.all(np.abs(got[~normal] - want[~normal]) <= np.spacing(np.float64(0.0)))  # subnormal results
    assert f(710.0) == np.inf and f(-746.0) == 0.0 and np.isnan(f(float("nan")))


@pytest.mark.parametrize("eos", [EOS_ION, EOS_PI])
def test_neutral_fraction_solves_the_equation_of_state(eos):
    """xi_n = get_neutral(T, rho) with T = (gamma-1)(e - (1-xi_n) chi)/(2 - xi_n),
    to the bisection's tolerance, over the whole cell array."""
    d = decks.partially_ionised(10, eos_number=eos)
    s = _sim(d)
    xi = s.get_field("xi_n")
    e = s.get_field("energy")
    rho = s.get_field("rho")
    p = d.params
    T = (p.gamma - 1.0) / (2.0 - xi) * (e - (1.0 - xi) * p.ionise_pot)
    c = decks.neutral_constants(eos)
    assert np.all((xi > 0.5) & (xi < 1.0))
    assert np.abs(xi - decks.get_neutral(T, rho, c)).max() < 1e-7


def _eta_perp_numpy(s, p, n):
    """neutral.f90:68-124 in numpy at the vertices 0:n."""
    rho, cv, e, xi = (s.get_field(k) for k in ("rho", "cv", "energy", "xi_n"))
    bx, by, bz = (s.get_field(k) for k in ("bx", "by", "bz"))
    # cell arrays start at -1, bx at (-2, -1, -1), by at (-1, -2, -1), bz at (-1, -1, -2)
    c = lambda a, i, j, k: a[1 + i:2 + n + i, 1 + j:2 + n + j, 1 + k:2 + n + k]
    fx = lambda i, j, k: bx[2 + i:3 + n + i, 1 + j:2 + n + j, 1 + k:2 + n + k]
    fy = lambda i, j, k: by[1 + i:2 + n + i, 2 + j:3 + n + j, 1 + k:2 + n + k]
    fz = lambda i, j, k: bz[1 + i:2 + n + i, 1 + j:2 + n + j, 2 + k:3 + n + k]
    o8 = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0), (0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 1)]
    rv = sum(c(rho, *o) * c(cv, *o) for o in o8) / sum(c(cv, *o) for o in o8)
    bxv = 0.25 * (fx(0, 0, 0) + fx(0, 1, 0) + fz(0, 0, 1) + fz(0, 1, 1))
    byv = 0.25 * (fy(0, 0, 0) + fy(1, 0, 0) + fz(0, 0, 1) + fz(1, 0, 1))
    bzv = 0.25 * (fz(0, 0, 0) + fz(1, 0, 0) + fz(0, 1, 0) + fz(1, 1, 0))
    tv = sum((c(e, *o) - (1.0 - c(xi, *o)) * p.ionise_pot) / (2.0 - c(xi, *o)) for o in o8) * (p.gamma - 1.0) / 8.0
    cst = dict(f_bar=p.f_bar, t_bar=p.t_bar, r_bar=p.r_bar, tr=p.tr)
    xv = decks.get_neutral(tv, rv, cst)
    f = np.maximum(1.0 - xv, np.finfo(np.float64).tiny)
    return np.minimum(p.eta_bar * xv / f * (bxv ** 2 + byv ** 2 + bzv ** 2) / rv ** 2 / np.sqrt(tv), 100.0)


def test_perpendicular_resistivity_matches_numpy():
    n = 10
    d = decks.partially_ionised(n, eta_bar=1e-2)
    s = _sim(d)
    ep = s.get_field("eta_perp")[1:n + 2, 1:n + 2, 1:n + 2]
    want = _eta_perp_numpy(s, d.params, n)
    assert want.max() > 1e-3
    assert np.allclose(ep, want, rtol=1e-12, atol=0.0)


@pytest.mark.parametrize("eos", [EOS_ION, EOS_PI])
def test_steps_conserve_mass_and_stay_finite(eos):
    n = 10
    d = decks.partially_ionised(n, eos_number=eos, eta_bar=1e-2)
    s = _sim(d)
    inner = (slice(2, n + 2),) * 3
    m0 = np.sum(s.get_field("rho")[inner] * s.get_field("cv")[inner])
    for k in range(1, 5):
        s.step(k)
    st = s.download()
    for f in STATE:
        assert np.isfinite(st[f]).all(), f
    m1 = np.sum(s.get_field("rho")[inner] * s.get_field("cv")[inner])
    assert abs(m1 - m0) <= 1e-12 * m0
    xi = s.get_field("xi_n")
    assert np.all((xi > 0.5) & (xi < 1.0))


def test_cowling_terms_add_heating():
    """eta_perp >= 0 adds (eta_perp + eta) |j_perp|^2 - eta |j_perp|^2 to
    the ohmic heating (lagran.F90:1564-1565)."""
    out = []
    for cow in (False, True):
        d = decks.partially_ionised(10, cowling=cow, eta_bar=1e-2)
        s = _sim(d)
        for k in range(1, 3):
            s.step(k)
        out.append(s.scalars().total_ohmic_heating)
    assert out[1] > out[0] > 0.0


@pytest.mark.parametrize("eos", [EOS_ION, EOS_PI])
def test_empty_temperature_bracket_is_an_error(eos):
    """A cell with negative energy has no temperature bracket: the reference
    stops (neutral.f90:171-174); the call returns LARE_EEOS."""
    d = decks.partially_ionised(8, eos_number=eos)
    d.state["energy"][5, 5, 5] = -1.0
    from oracle import oracle
    s = oracle.simulation(d)
    with pytest.raises(LareError) as ei:
        s.start(d.state)
    assert ei.value.code == -9


def test_ideal_eos_code_zero_is_ideal():
    """eos_number 0 (a zero-initialised struct) reads as EOS_IDEAL."""
    a = decks.blast(8)
    b = decks.blast(8, eos_number=0)
    ra, rb = _sim(a), _sim(b)
    for k in range(1, 3):
        ra.step(k)
        rb.step(k)
    for f in STATE:
        assert np.array_equal(ra.get_field(f), rb.get_field(f)), f


# ---------------------------------------------------------------------
# Optically thin radiation (radiative.f90), in the same file because it is
# the other per-cell energy source of lagran.F90:168-181.

def test_radiative_losses_constant_band_closed_form():
    """A static uniform plasma in a band where Q(T) is constant (pow = 0,
    0.562-1.995 MK) cools linearly: Townsend's exact step reduces to
    T' = T - dt time_norm (gamma-1)/2 rho rho_norm psi / (kb mf mh)."""
    from lare3d_b200.abi import State
    n = 8
    d = decks.radiative_blast(n, rho_norm=1.0e-9)
    p = d.params
    g = p.gamma
    T = 1.0e6
    e = T * 2.0 / (g - 1.0) / p.temp_norm
    st = State.zeros(n, n, n)
    st["rho"][...] = 1.0
    st["energy"][...] = e
    d.state = st
    s = _sim(d)
    _, dt = s.step(1)
    psi = 1e-13 * 10.0 ** -21.94
    kb, mh = 1.3806488e-23, 1.672621777e-27
    T1 = T - dt * p.time_norm * 0.5 * (g - 1.0) * 1.0 * p.rho_norm * psi / (kb * p.mf * mh)
    got = s.get_field("energy")[2:n + 2, 2:n + 2, 2:n + 2]
    want = T1 * 2.0 / (g - 1.0) / p.temp_norm
    assert T1 < 0.99 * T                     # a visible loss
    assert np.allclose(got, want, rtol=1e-9, atol=0.0)


def test_radiative_losses_cool_only_inside_the_table():
    """Cells below 2e4 K or above 1e7 K are left unchanged (the reference's
    CYCLE); cells inside lose energy, none gains."""
    n = 12
    d = decks.radiative_blast(n)
    d0 = decks.radiative_blast(n, radiation=0)
    s, s0 = _sim(d), _sim(d0)
    s.step(1)
    s0.step(1)
    e, e0 = s.get_field("energy"), s0.get_field("energy")
    p = d.params
    T = 0.5 * p.temp_norm * d.state["energy"] * (p.gamma - 1.0)
    inner = (slice(2, n + 2),) * 3
    inside = ((T > 2e4) & (T <= 1e7))[inner]
    assert np.all(e[inner] <= e0[inner] + 1e-15)
    assert np.all(e[inner][inside] < e0[inner][inside])


# ---------------------------------------------------------------------
# rke: the remap's kinetic-energy correction ([xyz]remap.f90, diagnostics.F90:613-629).

def test_rke_returns_the_remap_kinetic_energy_loss():
    """The momentum remap's dissipation is returned as heat: on the
    periodic Orszag-Tang vortex the total energy drifts by 4 % over ten
    steps without rke and by under 0.1 % with it; the correction only adds."""
    drift = []
    for rke in (0, 1):
        d = decks.orszag_tang(16, rke=rke)
        s = _sim(d)
        e0 = sum(s.energy()[:3])
        for k in range(1, 11):
            s.step(k)
        drift.append(abs(sum(s.energy()[:3]) - e0) / e0)
        if rke:
            assert s.get_field("delta_ke").min() >= 0.0
    assert drift[0] > 0.02 and drift[1] < 2e-3


def test_energy_correction_needs_rke():
    from oracle import oracle
    d = decks.blast(8)
    s = oracle.simulation(d)
    s.start(d.state)
    with pytest.raises(LareError):
        s.energy_correction()


# ---------------------------------------------------------------------
# cooling_term (lagran.F90:464-475, :1290-1302): moving averages of the
# heating taken off the energy.

def test_cooling_term_first_step_is_the_weighted_heating():
    """From zero averages, one Lagrangian step leaves cool_term_v =
    alpha_av dt visc_heat / rho exactly, and the energy lower than without."""
    n = 10
    out = {}
    for ct in (0, 1):
        d = decks.orszag_tang(n, cooling_term=ct, alpha_av=0.05)
        s = _sim(d)
        s.lagrangian_step(1)
        out[ct] = s
    s = out[1]
    dt = s.scalars().dt
    vh = s.get_field("visc_heat")[1:n + 1, 1:n + 1, 1:n + 1]        # 0:n+1 -> 1:n
    rho = s.get_field("rho")[2:n + 2, 2:n + 2, 2:n + 2]
    want = 0.05 * dt * vh / rho + (1.0 - 0.05) * 0.0
    assert np.array_equal(s.get_field("cool_term_v"), want)
    assert np.all(s.get_field("cool_term_b") >= 0.0) and s.get_field("cool_term_b").max() > 0.0
    inner = (slice(2, n + 2),) * 3
    assert s.get_field("energy")[inner].sum() < out[0].get_field("energy")[inner].sum()


# ---------------------------------------------------------------------
# The bounds-checked oracle build (every array access checked against the
# reference's Fortran bounds) over the widened physics, six steps each (all
# six Strang orderings of the remap).

@pytest.mark.parametrize("case", ["pip_all", "radiation_open"])
def test_widened_physics_bounds_checked(case):
    from lare3d_b200.abi import BC_OPEN
    from oracle import oracle
    if case == "pip_all":
        d = decks.partially_ionised(10, eta_bar=1e-2, rke=1, cooling_term=1, conduction=1, kappa_0=1e-2)
    else:
        d = decks.radiative_blast(10, rke=1, cooling_term=1, xbc_min=BC_OPEN, xbc_max=BC_OPEN)
    s = oracle.simulation(d, checked=True)
    s.start(d.state)
    for k in range(1, 7):
        s.step(k)
    st = s.download()
    for f in STATE:
        assert np.isfinite(st[f]).all(), f


# ---------------------------------------------------------------------
# coronal_heating: the user_defined_heating hook (lagran.F90:127).

def test_coronal_heating_adds_rate_times_previous_dt():
    """A static uniform plasma under a uniform heating rate gains exactly
    heat_in dt / rho in the first Lagrangian step, with the dt held before
    set_dt (the hook runs first); the reference's example rate is zero on
    the ghosts and positive inside."""
    from lare3d_b200.abi import State, alloc
    from oracle import oracle
    n = 8
    d = decks.blast(n, coronal_heating=1)
    st = State.zeros(n, n, n)
    st["rho"][...] = 2.0
    st["energy"][...] = 1.5
    d.state = st
    norm = decks.normalisation()
    ex = decks.example_heating(d, norm["time_norm"], norm["rho_norm"], 1.0e6)
    assert ex[0].max() == 0.0 and ex[2:n + 2, 2:n + 2, 2:n + 2].min() > 0.0
    heat = alloc("cell", n, n, n, 1.0e-3)
    s = oracle.simulation(d)
    s.upload(st)
    s.set_field("heat_in", heat)
    s.set_time(0.0, 0.01)
    s.boundary_conditions()
    s.eta_calc()
    s.lagrangian_step(1)
    inner = (slice(2, n + 2),) * 3
    want = 1.5 + heat[inner] * 0.01 / 2.0
    got = s.get_field("energy")[inner]
    assert heat[inner].max() > 0.0
    assert np.array_equal(got, want)


def test_radiative_losses_power_law_band_closed_form():
    """In the band where Q(T) = psi T^-2 (0.251-0.562 MK), dT/dt = -c psi T^-2
    integrates to T'^3 = T^3 - 3 c psi dt, with the c of the constant band;
    Townsend's exact step must reproduce it (its pow branch)."""
    from lare3d_b200.abi import State
    n = 8
    d = decks.radiative_blast(n, rho_norm=1.0e-11)
    p = d.params
    g = p.gamma
    T = 0.5e6
    st = State.zeros(n, n, n)
    st["rho"][...] = 1.0
    st["energy"][...] = T * 2.0 / (g - 1.0) / p.temp_norm
    d.state = st
    s = _sim(d)
    _, dt = s.step(1)
    psi = 1e-13 * 10.0 ** -10.4
    kb, mh = 1.3806488e-23, 1.672621777e-27
    c = p.time_norm * 0.5 * (g - 1.0) * 1.0 * p.rho_norm / (kb * p.mf * mh)
    T1 = (T ** 3 - 3.0 * c * psi * dt) ** (1.0 / 3.0)
    assert 0.251e6 < T1 < 0.999 * T                    # a visible loss inside the band
    got = s.get_field("energy")[2:n + 2, 2:n + 2, 2:n + 2]
    assert np.allclose(got, T1 * 2.0 / (g - 1.0) / p.temp_norm, rtol=1e-9, atol=0.0)
