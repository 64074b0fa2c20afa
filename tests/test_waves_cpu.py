"""Closed-form pins of the oracle: small-amplitude linear waves along each axis.

The reference ships no golden outputs for the step, so besides its own
invariants (tests/test_oracle_cpu.py) the oracle is held to the analytic
dispersion relation of the equations the reference solves.  On a periodic
box, with the shock viscosity off (visc1 = visc2 = 0, lagran.F90:532-857)
and no resistivity:

* a sound wave (rho = rho0 + d, p = p0 + c_s^2 d, v_a = c_s d / rho0 along
  the axis) travels at c_s = sqrt(gamma p0 / rho0) (the pressure of the
  ideal EOS, lagran.F90:91-97);
* an Alfven wave along a uniform field B0 on the axis (B_t = B0 e sin(k x),
  v_t = -v_A e sin(k x)) travels at v_A = B0 / sqrt(rho0): Lare's Lorentz
  force is j x B with j = curl B in normalised units (lagran.F90:330-375);
* a fast magnetosonic wave across a uniform transverse field B0 (rho and
  p as for sound, B_t = B0 (1 + d / rho0), v_a = v_f d / rho0) travels at
  v_f = sqrt(c_s^2 + v_A^2).

Each wave is run along x, y and z in turn (64 cells a wavelength along the
axis, 4 across) so that the three directional remaps (remap.f90:71-99 with
xremap.f90 / yremap.f90 / zremap.f90) and the staggering of every component
are exercised; the phase of the wave's Fourier mode gives its speed, which
must match the analytic one within 0.1 % (the scheme's measured dispersion
error at 64 cells a wavelength is 6e-6 for sound, 2e-4 for the Alfven
wave), the amplitude must be kept within 1 % after 0.3 periods (measured
0.9993), and the three axes must agree.
"""
import math

import numpy as np
import pytest

from lare3d_b200 import decks
from lare3d_b200.abi import State, default_params
from lare3d_b200.grid import grid

N_AX = 64       # cells per wavelength along the wave
N_TR = 4        # cells across
EPS = 1.0e-4    # relative amplitude
T_END = 0.3     # 0.3 wave periods at speed 1
GAMMA = 5.0 / 3.0
P0 = 0.6        # c_s = sqrt(gamma p0 / rho0) = 1 with rho0 = 1


def oracle_sim(deck):
    from oracle import oracle
    return oracle.simulation(deck)


def _deck(axis):
    n = [N_TR, N_TR, N_TR]
    n[axis] = N_AX
    dx = 1.0 / N_AX
    ext = [(0.0, N_TR * dx)] * 3
    ext[axis] = (0.0, 1.0)
    p = default_params(gamma=GAMMA, visc1=0.0, visc2=0.0, dt_multiplier=0.8)
    m = grid(n[0], n[1], n[2], ext[0], ext[1], ext[2])
    st = State.zeros(*n)
    return p, m, st, n


def _along(m, axis, kind):
    """The coordinate along the axis, shaped to broadcast over a 3-D array
    ('c' cell centres -1:n+2, 'b' nodes -2:n+2)."""
    key = "xyz"[axis] + kind
    shape = [1, 1, 1]
    shape[axis] = -1
    return m[key].reshape(shape)


def _phase_and_amplitude(prof, x):
    """prof = A sin(k x - phi): returns (phi in [0, 2 pi), A)."""
    k = 2.0 * math.pi
    s = float(np.sum(prof * np.sin(k * x)))
    c = float(np.sum(prof * np.cos(k * x)))
    phi = math.atan2(-c, s) % (2.0 * math.pi)
    amp = 2.0 / len(x) * math.hypot(s, c)
    return phi, amp


def _interior_profile(arr, axis):
    """Mean over the transverse axes of the interior points 1..n along each
    axis (array index i + 1 for Fortran index i on a cell-centred axis, whose
    extent is n + 4, and i + 2 on a node-centred one, extent n + 5)."""
    idx = []
    for a in range(3):
        n = N_AX if a == axis else N_TR
        off = 1 if arr.shape[a] == n + 4 else 2
        idx.append(slice(1 + off, 1 + off + n))
    others = tuple(a for a in range(3) if a != axis)
    return arr[tuple(idx)].mean(axis=others)


def wave_deck(kind, axis):
    """The periodic wave box of `kind` ("sound", "alfven", "fast") along
    `axis`: (deck, analytic speed, field whose mode is measured, its
    background value)."""
    p, m, st, n = _deck(axis)
    k = 2.0 * math.pi
    cs = math.sqrt(GAMMA * P0 / 1.0)
    b0 = 1.0
    va = b0 / math.sqrt(1.0)
    xc = _along(m, axis, "c")
    xb = _along(m, axis, "b")
    t_ax = (axis + 1) % 3  # the transverse component
    va_name = "vx vy vz".split()[axis]
    bt = "bx by bz".split()[t_ax]
    if kind == "alfven":
        st["rho"][...] = 1.0
        st["energy"][...] = P0 / ((GAMMA - 1.0) * 1.0)
        st["bx by bz".split()[axis]][...] = b0
        # the transverse component's faces are cell-centred along the wave axis
        st[bt][...] = np.broadcast_to(b0 * EPS * np.sin(k * xc), st[bt].shape)
        vt = "vx vy vz".split()[t_ax]
        st[vt][...] = np.broadcast_to(-va * EPS * np.sin(k * xb), st[vt].shape)
        speed, probe, base = va, bt, 0.0
    else:
        drho = EPS * np.sin(k * xc)
        rho = 1.0 + drho
        st["rho"][...] = np.broadcast_to(rho, st["rho"].shape)
        st["energy"][...] = np.broadcast_to((P0 + cs * cs * drho) / ((GAMMA - 1.0) * rho), st["energy"].shape)
        if kind == "fast":
            st[bt][...] = np.broadcast_to(b0 * (1.0 + drho), st[bt].shape)
            speed = math.sqrt(cs * cs + va * va)
        else:
            speed = cs
        st[va_name][...] = np.broadcast_to(speed * EPS * np.sin(k * xb), st[va_name].shape)
        probe, base = "rho", 1.0
    d = decks.Deck("wave_" + kind, p, n[0], n[1], n[2], m, st, nsteps=0)
    return d, speed, probe, base


def run_to_end(s):
    """Steps from t = 0 until t >= T_END, as the main loop of lare3d.f90:80-89."""
    t, step = 0.0, 0
    while t < T_END and step < 1000:
        t, _ = s.step(step)
        step += 1
    return t


def measured_mode(s, d, axis, probe, base):
    """(phase, amplitude) of the probe field's Fourier mode along the axis."""
    x = d.metrics["xyz"[axis] + "c"][2:2 + N_AX]
    return _phase_and_amplitude(_interior_profile(s.get_field(probe), axis) - base, x)


def _oracle_wave(kind, axis):
    d, speed, probe, base = wave_deck(kind, axis)
    s = oracle_sim(d)
    s.start(d.state)
    t = run_to_end(s)
    assert 0.28 <= t <= 0.32
    phi, amp = measured_mode(s, d, axis, probe, base)
    assert abs(phi / (2.0 * math.pi * t) / speed - 1.0) < 1e-3, (phi / (2.0 * math.pi * t), speed)
    assert 0.99 * EPS < amp <= 1.001 * EPS, amp
    return s, d, speed, phi, amp


def _node_mode(s, d, axis, name, sign=1.0):
    xb = d.metrics["xyz"[axis] + "b"][3:3 + N_AX]
    return _phase_and_amplitude(sign * _interior_profile(s.get_field(name), axis), xb)


@pytest.mark.parametrize("axis", [0, 1, 2], ids=["x", "y", "z"])
def test_sound_wave_speed(built, axis):
    s, d, cs, phi, amp = _oracle_wave("sound", axis)
    # the velocity carries the same phase (a wave travelling one way)
    phv, ampv = _node_mode(s, d, axis, "vx vy vz".split()[axis])
    assert abs(phv - phi) < 0.02 and abs(ampv / (cs * amp) - 1.0) < 0.02, (phv, phi, ampv)


@pytest.mark.parametrize("axis", [0, 1, 2], ids=["x", "y", "z"])
def test_alfven_wave_speed(built, axis):
    s, d, va, phi, amp = _oracle_wave("alfven", axis)
    phv, ampv = _node_mode(s, d, axis, "vx vy vz".split()[(axis + 1) % 3], sign=-1.0)
    assert abs(phv - phi) < 0.02 and abs(ampv / (va * amp) - 1.0) < 0.02, (phv, phi, ampv)
    # the density stays uniform to second order in the amplitude
    assert np.abs(s.get_field("rho")[2:-2, 2:-2, 2:-2] - 1.0).max() < 1e-6


@pytest.mark.parametrize("axis", [0, 1, 2], ids=["x", "y", "z"])
def test_fast_wave_speed(built, axis):
    s, d, vf, phi, amp = _oracle_wave("fast", axis)
    # the compressed transverse field moves with the density
    bt = "bx by bz".split()[(axis + 1) % 3]
    phb, ampb = measured_mode(s, d, axis, bt, 1.0)
    assert abs(phb - phi) < 0.02 and abs(ampb / amp - 1.0) < 0.02, (phb, phi, ampb)


def test_axes_agree(built):
    """The same wave along x, y and z gives the same profile to round-off."""
    for kind in ("sound", "alfven"):
        prof = []
        for axis in range(3):
            d, _, probe, _ = wave_deck(kind, axis)
            s = oracle_sim(d)
            s.start(d.state)
            run_to_end(s)
            prof.append(_interior_profile(s.get_field(probe), axis))
        assert np.abs(prof[1] - prof[0]).max() <= 1e-14 and np.abs(prof[2] - prof[0]).max() <= 1e-14, kind
