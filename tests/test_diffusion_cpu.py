"""Closed-form pins of the oracle: diffusive decay of a Fourier mode along each axis.

* Resistive diffusion (lagran.F90:1239-1635, eta_calc :1176-1230): with a
  uniform resistivity eta = eta_background and a weak transverse field
  B_t = e sin(k x) (no flow: the Lorentz force and the ohmic heating are of
  order e^2), dB/dt = -curl(eta curl B) = eta d2B/dx2, so the mode decays
  as exp(-eta k^2 t) through the full step with its resistive sub-cycles.
* Field-aligned conduction (conduct.f90:152-416): with B along the axis,
  the heat flux limiter off and the ideal EOS, the RKL2 update is
  rho de/dt = d/dx(kappa_0 T^(5/2) dT/dx) with T = (gamma - 1) e / 2
  (conduct.f90:72), so a small temperature mode on T0 decays at
  lambda = kappa_0 T0^(5/2) k^2 (gamma - 1) / (2 rho0) over one
  conduct_heat call.

The decay rates must match within 0.2 % (measured: -5.6e-4 resistive, and
-8.0e-4 for conduction, the second-order Laplacian's (k dx)^2 / 12 at 64
cells a wavelength), and the three axes must agree to round-off.
"""
import math

import numpy as np
import pytest

from lare3d_b200 import decks
from lare3d_b200.abi import State, default_params
from lare3d_b200.grid import grid
from test_waves_cpu import N_AX, N_TR, _along, _interior_profile, _phase_and_amplitude

EPS = 1.0e-4
GAMMA = 5.0 / 3.0
ETA = 1.0e-2
T_RES = 0.3
KAPPA = 1.0e-2
T0 = 1.0
DT_COND = 0.02


def oracle_sim(deck):
    from oracle import oracle
    return oracle.simulation(deck)


def _box(axis, **over):
    n = [N_TR, N_TR, N_TR]
    n[axis] = N_AX
    dx = 1.0 / N_AX
    ext = [(0.0, N_TR * dx)] * 3
    ext[axis] = (0.0, 1.0)
    p = default_params(gamma=GAMMA, visc1=0.0, visc2=0.0, dt_multiplier=0.8)
    for k, v in over.items():
        setattr(p, k, v)
    m = grid(n[0], n[1], n[2], ext[0], ext[1], ext[2])
    st = State.zeros(*n)
    return p, m, st, n


def resistive_deck(axis):
    """(deck, decay rate, probe field) of the resistive mode along `axis`."""
    p, m, st, n = _box(axis, resistive_mhd=1, eta_background=ETA, eta0=0.0, j_max=1.0e10)
    k = 2.0 * math.pi
    st["rho"][...] = 1.0
    st["energy"][...] = 0.6 / ((GAMMA - 1.0) * 1.0)
    bt = "bx by bz".split()[(axis + 1) % 3]
    # the transverse component's faces are cell-centred along the mode's axis
    st[bt][...] = np.broadcast_to(EPS * np.sin(k * _along(m, axis, "c")), st[bt].shape)
    return decks.Deck("resistive_mode", p, n[0], n[1], n[2], m, st, nsteps=0), ETA * k * k, bt


def conduction_deck(axis):
    """(deck, decay rate) of the temperature mode along `axis` with B along it."""
    p, m, st, n = _box(axis, conduction=1, kappa_0=KAPPA, heat_flux_limiter=0)
    k = 2.0 * math.pi
    st["rho"][...] = 1.0
    temp = T0 * (1.0 + EPS * np.sin(k * _along(m, axis, "c")))
    st["energy"][...] = np.broadcast_to(2.0 * temp / (GAMMA - 1.0), st["energy"].shape)
    st["bx by bz".split()[axis]][...] = 1.0
    lam = KAPPA * T0 ** 2.5 * k * k * (GAMMA - 1.0) / 2.0
    return decks.Deck("conduction_mode", p, n[0], n[1], n[2], m, st, nsteps=0), lam


def mode(s, d, axis, name, base=0.0):
    x = d.metrics["xyz"[axis] + "c"][2:2 + N_AX]
    return _phase_and_amplitude(_interior_profile(s.get_field(name), axis) - base, x)


def run_resistive(s, t_end=T_RES):
    """Steps until t >= t_end, as the main loop of lare3d.f90:80-89."""
    t, step = 0.0, 0
    while t < t_end and step < 1000:
        t, _ = s.step(step)
        step += 1
    return t


@pytest.mark.parametrize("axis", [0, 1, 2], ids=["x", "y", "z"])
def test_resistive_decay(built, axis):
    d, lam, bt = resistive_deck(axis)
    s = oracle_sim(d)
    s.start(d.state)
    t = run_resistive(s)
    assert s.scalars().peak_substeps >= 2  # the resistive sub-cycles ran
    phi, amp = mode(s, d, axis, bt)
    rate = -math.log(amp / EPS) / t
    assert abs(rate / lam - 1.0) < 2e-3, (rate, lam)
    assert min(phi, 2.0 * math.pi - phi) < 1e-6  # the mode does not move


@pytest.mark.parametrize("axis", [0, 1, 2], ids=["x", "y", "z"])
def test_conduction_decay(built, axis):
    d, lam = conduction_deck(axis)
    s = oracle_sim(d)
    s.start(d.state)
    stages = s.conduct_heat(DT_COND)
    assert stages >= 2
    phi, amp = mode(s, d, axis, "energy", 2.0 * T0 / (GAMMA - 1.0))
    rate = -math.log(amp / (2.0 * T0 * EPS / (GAMMA - 1.0))) / DT_COND
    assert abs(rate / lam - 1.0) < 2e-3, (rate, lam)
    assert min(phi, 2.0 * math.pi - phi) < 1e-6


def test_diffusion_axes_agree(built):
    for build in (lambda a: resistive_deck(a)[0], lambda a: conduction_deck(a)[0]):
        prof = []
        for axis in range(3):
            d = build(axis)
            s = oracle_sim(d)
            s.start(d.state)
            if d.name == "resistive_mode":
                run_resistive(s)
                name = "bx by bz".split()[(axis + 1) % 3]
            else:
                s.conduct_heat(DT_COND)
                name = "energy"
            prof.append(_interior_profile(s.get_field(name), axis))
        assert np.abs(prof[1] - prof[0]).max() <= 1e-15 and np.abs(prof[2] - prof[0]).max() <= 1e-15, d.name
