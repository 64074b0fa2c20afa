"""Closed-form pins of the oracle's gravity (lagran.F90:379).

The momentum update adds -rho_v grav(iz) to the vertical force of vertex
(ix, iy, iz), grav being a profile over the vertices' z index, and divides
the force by rho_v (:382-384):

* free fall: a uniform state in a periodic box falls as a whole, every
  vertex at vz = -g t to round-off (measured 8.9e-16), while the remap
  carries the uniform density and energy through the box unchanged;
* hydrostatic balance: between walls (BC_USER: no flow through them,
  mirrored cells) an isothermal atmosphere whose cell densities satisfy the
  scheme's discrete balance at every interior vertex,

      p(iz+1) - p(iz) = -dzc(iz) grav(iz) rho_v(iz),
      rho_v(iz) = (rho(iz) dzb(iz) + rho(iz+1) dzb(iz+1)) / (dzb(iz) + dzb(iz+1)),

  (the pressure force of :279-283 with the vertex density of :99-121) stays
  at rest to round-off for two sound crossings (measured 1.7e-14), both for
  uniform gravity and for a profile varying by half along the box.  The pin
  is sharp: the same construction with grav taken one vertex up moves at
  6.6e-3, and the continuum isothermal profile rho = exp(-g z / c^2), off the
  discrete balance by O(dz^2), at 7.6e-6.
"""
import math

import numpy as np
import pytest

from lare3d_b200 import decks
from lare3d_b200.abi import BC_PERIODIC, BC_USER, State, default_params
from lare3d_b200.grid import grid

NZ = 64
NT = 4
GAMMA = 5.0 / 3.0
C2 = 1.0      # isothermal p / rho
G0 = 1.0      # scale height c^2 / g = 1, the box height


def oracle_sim(deck):
    from oracle import oracle
    return oracle.simulation(deck)


def gravity_profile(m, kind):
    """grav over vertices -1..nz+2."""
    zb = m["zb"][1:]
    if kind == "uniform":
        return np.full(NZ + 4, G0)
    return G0 * (1.0 + 0.5 * np.sin(2.0 * math.pi * zb))


def atmosphere(kind, balance="discrete", shift=0):
    """(deck, grav) of an isothermal atmosphere between walls in z.  Cell
    arrays run over -1..nz+2 and vertex arrays over -2..nz+2; dzb over
    -1..nz+2 and dzc over -1..nz+1."""
    dz = 1.0 / NZ
    bcs = (BC_PERIODIC, BC_PERIODIC, BC_USER)
    p = default_params(gamma=GAMMA, visc1=0.0, visc2=0.0, dt_multiplier=0.8)
    p.zbc_min = BC_USER
    p.zbc_max = BC_USER
    m = grid(NT, NT, NZ, (0.0, NT * dz), (0.0, NT * dz), (0.0, 1.0), bcs=bcs)
    g = gravity_profile(m, kind)
    dzb, dzc, zc = m["dzb"], m["dzc"], m["zc"]
    rho = np.empty(NZ + 4)
    rho[2] = 1.0                        # cell 1
    for iz in range(1, NZ):             # vertex iz, between cells iz and iz + 1
        if balance == "discrete":
            b1, b2 = dzb[iz + 1], dzb[iz + 2]
            w1, w2 = b1 / (b1 + b2), b2 / (b1 + b2)
            gz = g[iz + 1 + shift]
            rho[iz + 2] = rho[iz + 1] * (C2 - dzc[iz + 1] * gz * w1) / (C2 + dzc[iz + 1] * gz * w2)
        else:
            rho[iz + 2] = math.exp(-G0 * (zc[iz + 2] - zc[2]) / C2)
    rho[:2] = rho[2]                    # the ghosts, which the walls mirror at start
    rho[-2:] = rho[-3]
    st = State.zeros(NT, NT, NZ)
    st["rho"][...] = rho[None, None, :]
    st["energy"][...] = C2 / (GAMMA - 1.0)
    return decks.Deck("atmosphere", p, NT, NT, NZ, m, st, nsteps=0), g


def settle(kind, balance="discrete", shift=0, steps=200):
    """(largest |v|, largest relative density change) after `steps` steps."""
    d, g = atmosphere(kind, balance, shift)
    s = oracle_sim(d)
    s.start(d.state, grav=g)
    t = 0.0
    for step in range(steps):
        t, _ = s.step(step)
    assert t > 1.9  # two sound crossings of the box
    v = max(float(np.abs(s.get_field(c)).max()) for c in ("vx", "vy", "vz"))
    r = s.get_field("rho")[2:-2, 2:-2, 2:-2]
    r0 = d.state["rho"][2:-2, 2:-2, 2:-2]
    return v, float(np.abs(r / r0 - 1.0).max())


def test_free_fall(built):
    n, g = 16, 0.7
    p = default_params(visc1=0.0, visc2=0.0, dt_multiplier=0.8)
    m = grid(n, n, n, (0.0, 1.0), (0.0, 1.0), (0.0, 1.0))
    st = State.zeros(n, n, n)
    st["rho"][...] = 1.3
    st["energy"][...] = 1.0 / ((p.gamma - 1.0) * 1.3)
    d = decks.Deck("free_fall", p, n, n, n, m, st, nsteps=0)
    s = oracle_sim(d)
    s.start(d.state, grav=np.full(n + 4, g))
    dts = [s.step(step)[1] for step in range(40)]
    t = math.fsum(dts)
    assert t > 1.5  # the box has fallen more than its own height
    vz = s.get_field("vz")[2:-2, 2:-2, 2:-2]
    assert np.abs(vz / (-g * t) - 1.0).max() < 1e-14
    assert np.abs(s.get_field("vx")).max() == 0.0 and np.abs(s.get_field("vy")).max() == 0.0
    assert np.ptp(s.get_field("rho")) == 0.0 and np.ptp(s.get_field("energy")) == 0.0


@pytest.mark.parametrize("kind", ["uniform", "varying"])
def test_hydrostatic_balance_holds(built, kind):
    v, dr = settle(kind)
    assert v < 1e-12 and dr < 1e-12, (v, dr)


def test_hydrostatic_balance_is_sharp(built):
    v_shift, _ = settle("varying", shift=1)
    assert v_shift > 1e-3, v_shift
    v_cont, _ = settle("uniform", balance="continuum")
    assert 1e-6 < v_cont < 1e-4, v_cont
