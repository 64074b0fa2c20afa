"""Closed-form pin of the oracle's viscous damping (lagran.F90:483-524).

With use_viscous_damping each step adds dt visc3 (discrete Laplacian of v)
to every vertex velocity 0..n, before the shock viscosity and set_dt
(lagran.F90:129-131).  A shear mode, one velocity component
v_c = eps sin(4 pi x_a) varying along another axis a, in a periodic box of
uniform density and pressure with no field and the shock viscosity off, is
divergence-free: no other force acts on it, and the Laplacian's eigenvalue
lam = (4 / dx^2) sin^2(2 pi dx) gives each step's factor 1 - dt visc3 lam.

Three properties of the reference's order are pinned with it:

* the first step does not damp: dt is zero until the first set_dt, which
  comes after viscous_damping;
* no velocity ghost is refreshed between viscous_damping and the predictor
  (lagran.F90:129-183), so the ghost vertices beyond the box faces normal to
  the component keep the undamped velocity for that step.  The ghost cells
  between a stale and a damped vertex change volume in
  b_field_and_cv1_update, and their pressure pushes back on the face vertices
  with about a third of the damping force (measured 0.31 of it on the face
  layer and 0.24 on its edges, at 32 to 128 cells alike), while every vertex
  two or more layers from those faces takes the exact factor to round-off;
* over many steps the mode therefore decays at 1 - 0.31 / NT of the viscous
  rate (NT layers across, one of them the face layer; measured 0.951 at
  NT = 6), not at the full rate, and sheds a small compressive wave that
  falls with the cell size.

set_dt has no visc3 limit (lagran.F90:1070-1166): the explicit damping is
stable only while dt visc3 (4/dx^2 + 4/dy^2 + 4/dz^2) < 2, which the
decks here keep below 1.
"""
import math

import numpy as np
import pytest

from lare3d_b200 import decks
from lare3d_b200.abi import State, alloc, default_params
from lare3d_b200.grid import grid

NT = 6             # vertex layers 0..NT across the mode
EPS = 1e-6         # small enough that the mode's own nonlinearity is below 1e-6 of it
MODE = 2           # wavelengths in the unit box
VISC3 = 2e-3
AXES = [(0, 1), (1, 2), (2, 0)]   # (axis of variation, velocity component)


def shear_deck(n_along, axis, comp):
    n = [NT, NT, NT]
    n[axis] = n_along
    dx = 1.0 / n_along
    ext = [(0.0, NT * dx)] * 3
    ext[axis] = (0.0, 1.0)
    p = default_params(dt_multiplier=0.8, visc1=0.0, visc2=0.0, use_viscous_damping=1)
    m = grid(n[0], n[1], n[2], *ext)
    st = State.zeros(*n)
    st["rho"][...] = 1.0
    st["energy"][...] = 1.0 / (p.gamma - 1.0)  # p = 1
    shape = [1, 1, 1]
    shape[axis] = -1
    xb = m["xyz"[axis] + "b"].reshape(shape)
    v = "vx vy vz".split()[comp]
    st[v][...] = np.broadcast_to(EPS * np.sin(2.0 * math.pi * MODE * xb), st[v].shape)
    return decks.Deck("shear_damping", p, n[0], n[1], n[2], m, st, nsteps=0)


def eigenvalue(n_along):
    dx = 1.0 / n_along
    return 4.0 / (dx * dx) * math.sin(math.pi * MODE * dx) ** 2


def start(d, visc3=VISC3):
    from oracle import oracle
    s = oracle.simulation(d)
    s.start(d.state, visc3=alloc("node", d.nx, d.ny, d.nz, visc3))
    return s


def component(s, comp):
    """Vertices 0..n of one velocity component (vertex fields start at -2)."""
    return s.get_field("vx vy vz".split()[comp])[2:-2, 2:-2, 2:-2]


@pytest.mark.parametrize("axis,comp", AXES, ids=["vy(x)", "vz(y)", "vx(z)"])
def test_one_step_of_damping(built, axis, comp):
    n_along = 32
    d = shear_deck(n_along, axis, comp)
    s = start(d)
    v0 = component(s, comp)
    _, dt0 = s.step(0)
    v1 = component(s, comp)
    assert np.abs(v1 - v0).max() <= 1e-15 * EPS  # dt = 0 before the first set_dt
    s.step(1)
    v2 = component(s, comp)
    a = dt0 * VISC3 * eigenvalue(n_along)
    assert dt0 * VISC3 * 12.0 * n_along ** 2 < 1.0  # explicit stability, all three axes
    dev = np.moveaxis((v2 - (1.0 - a) * v1) / (EPS * a), comp, 0)
    layer = np.abs(dev).reshape(NT + 1, -1).max(axis=1)
    # two or more layers from the faces normal to the component: exact (measured 3.5e-14)
    assert layer[2:NT - 1].max() <= 1e-11, layer
    # next to them: the remap's reconstruction across the face (measured 2e-7)
    assert layer[1] <= 1e-5 and layer[NT - 1] <= 1e-5, layer
    # the face layers: the stale ghosts' pushback (measured 0.31 of the damping)
    for f in (0, NT):
        assert 0.2 <= layer[f] <= 0.4, layer
        face = np.moveaxis(v1, comp, 0)[f]
        assert np.sum(dev[f] * face) > 0.0  # damped less than the factor says


def test_shear_mode_decays_at_the_face_reduced_rate(built):
    n_along = 64
    d = shear_deck(n_along, 0, 1)
    s = start(d)
    t, step, dts = 0.0, 0, []
    while t < 1.0 and step < 1000:
        t, dt = s.step(step)
        dts.append(dt)
        step += 1
    x = d.metrics["xb"][2:2 + n_along + 1]
    sn = np.sin(2.0 * math.pi * MODE * x)
    v = component(s, 1)
    amp = np.tensordot(sn, v, axes=(0, 0)).mean() / np.dot(sn, sn) / EPS
    # each step damps with the previous step's dt; the last dt is not used yet
    t_damped = math.fsum(dts[:-1])
    rate = -math.log(amp) / (t_damped * VISC3 * eigenvalue(n_along))
    assert abs(rate - (1.0 - 0.31 / NT)) < 0.01, rate  # measured 0.951
    assert amp < 0.75  # the mode lost a quarter of its amplitude
    # the shear stays a shear: the shed compression is below 1e-3 of the mode
    assert np.abs(component(s, 0)).max() < 1e-3 * EPS
    assert np.abs(s.get_field("rho")[2:-2, 2:-2, 2:-2] - 1.0).max() < 1e-3 * EPS


def test_damped_shear_axes_agree(built):
    """The three cyclic permutations of the problem give the same profile.  The
    remap's sweep order cycles with the step (remap.f90:71-98), so the permuted
    problems see the orders in another sequence, and the compressive part
    (1e-3 of the mode) differs at splitting order: agreement to 1e-10 of the
    amplitude (measured 1.0e-10) rather than round-off."""
    n_along = 32
    prof = []
    for axis, comp in AXES:
        d = shear_deck(n_along, axis, comp)
        s = start(d)
        t, step = 0.0, 0
        while t < 1.0 and step < 1000:
            t, _ = s.step(step)
            step += 1
        v = np.moveaxis(component(s, comp), axis, 0)
        prof.append(v.reshape(n_along + 1, -1).mean(axis=1) / EPS)
    assert np.abs(prof[1] - prof[0]).max() <= 5e-10 and np.abs(prof[2] - prof[0]).max() <= 5e-10
