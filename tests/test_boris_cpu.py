"""Closed-form pin of the oracle's Boris correction (boris = 1).

Where the Alfven speed v_A^2 = B^2 / rho reaches va_max, set_dt
(lagran.F90:1092-1109) sets gamma_boris = 1 / (1 + v_A^2 / va_max^2), which
scales the Lorentz force of the momentum update (:375-377), the fast speed of
the shock viscosity (:556) and the time step's signal speed (:1109).  The
linear waves of tests/test_waves_cpu.py then travel at the limited speeds

    c_A^2 = gamma_boris v_A^2,      c_f^2 = c_s^2 + gamma_boris v_A^2,

and each starts from its eigenvector at that speed (v_t = -c_A B_t / B0 for
the Alfven wave, v = c_f drho / rho0 for the fast wave), or it splits into
two counter-running waves.  With v_A = 1 and c_s = 1:

* va_max = 0.8 and 0.5 (gamma_boris 0.390 and 0.2): the Alfven wave runs
  at 0.6247 and 0.4472 (measured within 4.4e-4, bar 1e-3), the fast wave at
  1.1791 and 1.0954 (measured within 2.3e-5), both keeping their amplitude
  within 1 %, on every axis;
* va_max = 1.2, above v_A: gamma_boris stays 1 and the Alfven wave runs at
  v_A (the switch of :1106);
* the first step's dt is 0.8 dx / sqrt(c_s^2 + gamma_boris v_A^2), the time
  step's signal speed limited the same way (within 1e-7 for the Alfven
  wave, whose |B| changes at second order in its amplitude, and 2.9e-5 for
  the fast wave, whose signal speed changes at first order).
"""
import math

import pytest

import test_waves_cpu as waves

VA = 1.0
CS2 = waves.GAMMA * waves.P0


def gamma_boris(va_max):
    return 1.0 / (1.0 + VA * VA / (va_max * va_max)) if VA >= va_max else 1.0


def limited_speed(kind, va_max):
    g = gamma_boris(va_max)
    return math.sqrt(g) * VA if kind == "alfven" else math.sqrt(CS2 + g * VA * VA)


def boris_wave_deck(kind, axis, va_max):
    """The wave box of tests/test_waves_cpu.py with boris on and the velocity
    rescaled to the eigenvector at the limited speed."""
    d, speed, probe, base = waves.wave_deck(kind, axis)
    d.params.boris = 1
    d.params.va_max = va_max
    c = limited_speed(kind, va_max)
    v = "vx vy vz".split()[(axis + 1) % 3 if kind == "alfven" else axis]
    d.state[v][...] *= c / speed
    return d, c, probe, base


@pytest.mark.parametrize("va_max", [0.8, 0.5])
@pytest.mark.parametrize("kind", ["alfven", "fast"])
@pytest.mark.parametrize("axis", [0, 1, 2], ids=["x", "y", "z"])
def test_boris_limited_wave_speed(built, axis, kind, va_max):
    d, c, probe, base = boris_wave_deck(kind, axis, va_max)
    s = waves.oracle_sim(d)
    s.start(d.state)
    t, dt0 = s.step(0)
    dx = 1.0 / waves.N_AX
    want_dt = d.params.dt_multiplier * dx / math.sqrt(CS2 + gamma_boris(va_max) * VA * VA)
    # the Alfven wave changes |B| at second order in its amplitude, the fast
    # wave the signal speed at first order (measured 2.9e-5 of dt)
    bar = 1e-7 if kind == "alfven" else 0.5 * waves.EPS
    assert abs(dt0 / want_dt - 1.0) < bar, (dt0, want_dt)
    step = 1
    while t < waves.T_END and step < 1000:
        t, _ = s.step(step)
        step += 1
    phi, amp = waves.measured_mode(s, d, axis, probe, base)
    assert abs(phi / (2.0 * math.pi * t) / c - 1.0) < 1e-3, (phi / (2.0 * math.pi * t), c)
    assert 0.99 * waves.EPS < amp <= 1.001 * waves.EPS, amp


def test_boris_off_below_the_limit(built):
    d, c, probe, base = boris_wave_deck("alfven", 0, 1.2)
    assert c == VA
    s = waves.oracle_sim(d)
    s.start(d.state)
    t = waves.run_to_end(s)
    phi, _ = waves.measured_mode(s, d, 0, probe, base)
    assert abs(phi / (2.0 * math.pi * t) - VA) < 1e-3 * VA
