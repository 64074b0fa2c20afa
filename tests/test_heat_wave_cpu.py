"""Closed-form pin of the oracle's nonlinear conduction: the planar Zel'dovich heat wave.

tests/test_diffusion_cpu.py pins the conductivity at one temperature.  Here
its temperature dependence is pinned: with B along the axis, the heat flux
limiter off and uniform density, the RKL2 update (conduct.f90:152-416) solves
T_t = a (T^n T_x)_x with n = 5/2 and a = kappa_0 (gamma - 1) / (2 rho)
(T = (gamma - 1) e / 2, conduct.f90:72), whose planar self-similar solution
from a concentrated release (Zel'dovich and Raizer; Barenblatt) is

    T(x, t) = tau^-alpha (C - k x^2 tau^-2alpha)_+^(1/n),
    tau = a t / (n + 1), alpha = 1 / (n + 2), k = alpha n / (2 (n + 1)),

a wave with a sharp front at x_f = (C / k)^(1/2) tau^alpha.  The box starts from
the solution at tau_0 (front at 0.15, on a background 1e-6) and is advanced
by sixty conduct_heat calls to the time at which the front reaches 0.5, 256
cells along the axis.  The central temperature must be within 0.5 % of the
exact one (measured 0.1 %), the mean error within 0.3 % of it (measured
0.11 %; the largest error, 8 %, sits at the front, where the exact profile's
slope is infinite), the front at 20 % and 50 % of the central temperature
within one cell (measured 0.4 and 0.1 cells), the total energy conserved to
round-off (the fluxes are differences of face fluxes), and the three axes
must give the same profile to round-off.
"""
import math

import numpy as np
import pytest

from lare3d_b200 import decks
from lare3d_b200.abi import State, default_params
from lare3d_b200.grid import grid

NW = 256          # cells along the wave
NT = 4            # cells across
LW = 2.0          # box length along the wave, centred on the release
N_EXP = 2.5       # T^(5/2) conductivity (conduct.f90:27)
ALPHA = 1.0 / (N_EXP + 2.0)
KW = ALPHA * N_EXP / (2.0 * (N_EXP + 1.0))
GAMMA = 5.0 / 3.0
RHO = 1.0
KAPPA = 3.0       # a = kappa (gamma - 1) / (2 rho) = 1
A_DIFF = KAPPA * (GAMMA - 1.0) / (2.0 * RHO)
TAU0 = 0.02
XF0, XF1 = 0.15, 0.5
C_W = KW * (XF0 / TAU0 ** ALPHA) ** 2
TAU1 = TAU0 * (XF1 / XF0) ** (1.0 / ALPHA)
SUBSTEPS = 60
T_BACKGROUND = 1.0e-6


def wave_temperature(x, tau):
    return tau ** (-ALPHA) * np.maximum(C_W - KW * x * x * tau ** (-2.0 * ALPHA), 0.0) ** (1.0 / N_EXP)


def heat_wave_deck(axis):
    n = [NT, NT, NT]
    n[axis] = NW
    dx = LW / NW
    ext = [(0.0, NT * dx)] * 3
    ext[axis] = (-0.5 * LW, 0.5 * LW)
    p = default_params(gamma=GAMMA, conduction=1, kappa_0=KAPPA, heat_flux_limiter=0)
    m = grid(n[0], n[1], n[2], ext[0], ext[1], ext[2])
    st = State.zeros(*n)
    shape = [1, 1, 1]
    shape[axis] = -1
    xc = m["xyz"[axis] + "c"].reshape(shape)
    temp = wave_temperature(xc, TAU0) + T_BACKGROUND
    st["rho"][...] = RHO
    st["energy"][...] = np.broadcast_to(2.0 * temp / (GAMMA - 1.0), st["energy"].shape)
    st["bx by bz".split()[axis]][...] = 1.0
    return decks.Deck("heat_wave", p, n[0], n[1], n[2], m, st, nsteps=0)


def advance(s):
    """The wave from tau_0 to tau_1 in SUBSTEPS conduct_heat calls."""
    dt = (TAU1 - TAU0) * (N_EXP + 1.0) / A_DIFF / SUBSTEPS
    return [s.conduct_heat(dt) for _ in range(SUBSTEPS)]


def wave_profile(energy, axis):
    """Temperature of cells 1..NW along the wave, averaged across it."""
    idx = [slice(2, 2 + NT)] * 3
    idx[axis] = slice(2, 2 + NW)
    others = tuple(a for a in range(3) if a != axis)
    return (GAMMA - 1.0) / 2.0 * energy[tuple(idx)].mean(axis=others)


def front(x, temp, frac):
    """Where temp falls through frac of its maximum, right of the centre."""
    tc = temp.max()
    i = np.nonzero((x > 0.0) & (temp < frac * tc))[0][0]
    return x[i - 1] + (temp[i - 1] - frac * tc) / (temp[i - 1] - temp[i]) * (x[i] - x[i - 1])


def wave_errors(x, temp):
    """(central temperature error, mean error, front errors in cells), relative to T_c."""
    exact = wave_temperature(x, TAU1)
    tc = exact.max()
    dx = LW / NW
    fronts = [(front(x, temp, f) - front(x, exact, f)) / dx for f in (0.2, 0.5)]
    return abs(temp.max() / tc - 1.0), float(np.mean(np.abs(temp - exact))) / tc, fronts


def oracle_sim(deck):
    from oracle import oracle
    return oracle.simulation(deck)


@pytest.mark.parametrize("axis", [0, 1, 2], ids=["x", "y", "z"])
def test_heat_wave_matches_the_similarity_solution(built, axis):
    d = heat_wave_deck(axis)
    s = oracle_sim(d)
    s.start(d.state)
    e0 = math.fsum(d.state["energy"][2:-2, 2:-2, 2:-2].ravel())
    stages = advance(s)
    assert min(stages) >= 2
    energy = s.get_field("energy")
    assert abs(math.fsum(energy[2:-2, 2:-2, 2:-2].ravel()) / e0 - 1.0) < 1e-12
    x = d.metrics["xyz"[axis] + "c"][2:2 + NW]
    dtc, l1, fronts = wave_errors(x, wave_profile(energy, axis))
    assert dtc < 5e-3, dtc
    assert l1 < 3e-3, l1
    assert max(abs(f) for f in fronts) < 1.0, fronts


def test_heat_wave_axes_agree(built):
    prof = []
    for axis in range(3):
        d = heat_wave_deck(axis)
        s = oracle_sim(d)
        s.start(d.state)
        advance(s)
        prof.append(wave_profile(s.get_field("energy"), axis))
    assert np.abs(prof[1] - prof[0]).max() <= 1e-14 and np.abs(prof[2] - prof[0]).max() <= 1e-14
