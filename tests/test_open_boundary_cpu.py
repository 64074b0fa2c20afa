"""The oracle's open (characteristic) boundary measured by a sound pulse.

A right- or left-running acoustic pulse (Gaussian, amplitude 1e-3 of the
background, half-width 0.05) in a tube of 256 cells along one axis, open
at both ends (BC_OPEN, openboundary.f90:30-323, the ghosts holding the
background as the far field), periodic across, shock viscosity off.  After
the pulse has met the face (c_s t = 0.8 from the middle of the tube) what
is left in the tube is its reflection:

* the open faces return 0.283 of the pulse's amplitude, on all six faces
  alike, as a compression at the mirror position (a partly rigid face);
  a wall (BC_USER) returns all of it;
* the cause is in the reference's order, not in the characteristic
  solver: velocity_bcs (boundary.f90:255-295) fills the velocity ghosts of
  BC_USER faces only, so on an open face the ghost vertices keep the
  far-field velocity and the ghost cell between them and the boundary
  vertex is squeezed like a wall's.  A scratch copy of the oracle that
  copies the boundary vertex's velocity into the first ghost vertex
  returns 0.0035 of the pulse instead.  The engines reproduce the
  reference's behaviour; nothing here changes it.
"""
import math

import numpy as np
import pytest

from lare3d_b200 import decks
from lare3d_b200.abi import BC_OPEN, BC_PERIODIC, BC_USER, State, default_params
from lare3d_b200.grid import grid

N = 256
NT = 4
GAMMA = 5.0 / 3.0
P0 = 0.6
EPS = 1.0e-3
WIDTH = 0.05
CS = math.sqrt(GAMMA * P0)


def pulse(x):
    return EPS * np.exp(-((x - 0.5) / WIDTH) ** 2)


def tube_deck(axis, bc, direction):
    n = [NT, NT, NT]
    n[axis] = N
    dx = 1.0 / N
    ext = [(0.0, NT * dx)] * 3
    ext[axis] = (0.0, 1.0)
    bcs = [BC_PERIODIC] * 3
    bcs[axis] = bc
    p = default_params(gamma=GAMMA, visc1=0.0, visc2=0.0, dt_multiplier=0.8)
    for side, name in enumerate("xyz"):
        setattr(p, name + "bc_min", bcs[side])
        setattr(p, name + "bc_max", bcs[side])
    m = grid(n[0], n[1], n[2], ext[0], ext[1], ext[2], bcs=tuple(bcs))
    st = State.zeros(*n)
    shape = [1, 1, 1]
    shape[axis] = -1
    xc = m["xyz"[axis] + "c"].reshape(shape)
    xb = m["xyz"[axis] + "b"].reshape(shape)
    drho = pulse(xc)
    rho = 1.0 + drho
    st["rho"][...] = np.broadcast_to(rho, st["rho"].shape)
    st["energy"][...] = np.broadcast_to((P0 + CS * CS * drho) / ((GAMMA - 1.0) * rho), st["energy"].shape)
    v = "vx vy vz".split()[axis]
    st[v][...] = np.broadcast_to(direction * CS * pulse(xb), st[v].shape)
    return decks.Deck("acoustic_pulse", p, n[0], n[1], n[2], m, st, nsteps=0)


def reflection(axis, bc, direction):
    """(amplitude left in the tube / EPS, its position, its sign, expected position)."""
    from oracle import oracle
    d = tube_deck(axis, bc, direction)
    s = oracle.simulation(d)
    s.start(d.state)
    t, step = 0.0, 0
    while t < 0.8 / CS and step < 5000:
        t, _ = s.step(step)
        step += 1
    idx = [slice(2, 2 + NT)] * 3
    idx[axis] = slice(2, 2 + N)
    others = tuple(a for a in range(3) if a != axis)
    r = s.get_field("rho")[tuple(idx)].mean(axis=others) - 1.0
    x = d.metrics["xyz"[axis] + "c"][2:2 + N]
    i = int(np.argmax(np.abs(r)))
    mirror = 2.0 - (0.5 + CS * t) if direction > 0 else -(0.5 - CS * t)
    return abs(r[i]) / EPS, x[i], math.copysign(1.0, r[i]), mirror


@pytest.mark.parametrize("direction", [1, -1], ids=["max-face", "min-face"])
@pytest.mark.parametrize("axis", [0, 1, 2], ids=["x", "y", "z"])
def test_open_face_reflects_a_fixed_fraction(built, axis, direction):
    amp, at, sign, mirror = reflection(axis, BC_OPEN, direction)
    assert 0.27 < amp < 0.30, amp          # measured 0.2828 on every face
    assert sign > 0.0                       # a compression returns as a compression
    assert abs(at - mirror) < 1.5 / N, (at, mirror)


def test_wall_reflects_the_whole_pulse(built):
    amp, at, sign, mirror = reflection(0, BC_USER, 1)
    assert amp > 0.99 and sign > 0.0, amp   # measured 0.9994
    assert abs(at - mirror) < 1.5 / N, (at, mirror)
