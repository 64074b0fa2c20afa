"""Closed-form pin of the oracle's nonlinear behaviour: Sod's shock tube along each axis.

The linear pins (tests/test_waves_cpu.py, tests/test_diffusion_cpu.py) run
with the shock viscosity off.  Here it is on (visc1 = 0.1, visc2 = 0.5, the
shipped deck's values, control.f90): a tube of 256 cells along one axis and
4 across, walls on both ends of the tube (BC_USER: mirrored density, energy
and B, no flow through the wall, boundary.f90), periodic across, gamma = 1.4,
left state (rho, p) = (1, 1), right state (0.125, 0.1), at rest, the
interface at the middle.  At t = 0.2 the waves are still clear of the walls,
and the solution is compared with the exact solution of the Riemann problem
(the iterative star-pressure solver of Toro, "Riemann Solvers and Numerical
Methods for Fluid Dynamics", ch. 4, restated here): the mean absolute
density error below 0.005 (measured 0.0034), the shock within 1.5 cells of
its exact position (measured 0.44 cells behind), the density of the plateau
between the contact and the shock within 0.005 of its exact 0.2656
(measured 0.0017), and the three axes giving the same profile to round-off.
"""
import math

import numpy as np
import pytest

from lare3d_b200 import decks
from lare3d_b200.abi import BC_PERIODIC, BC_USER, State, default_params
from lare3d_b200.grid import grid

N = 256
NT = 4
GAMMA = 1.4
T_END = 0.2
LEFT = (1.0, 0.0, 1.0)     # rho, u, p
RIGHT = (0.125, 0.0, 0.1)


def exact_riemann(left, right, g, xi):
    """Density, velocity and pressure of the exact Riemann solution at the
    similarity coordinates xi = (x - x0) / t."""
    dl, ul, pl = left
    dr, ur, pr = right
    cl, cr = math.sqrt(g * pl / dl), math.sqrt(g * pr / dr)

    def fk(p, dk, pk, ck):  # the pressure function of one side and its derivative
        if p > pk:  # shock
            a, b = 2.0 / ((g + 1.0) * dk), (g - 1.0) / (g + 1.0) * pk
            q = math.sqrt(a / (p + b))
            return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (b + p))
        r = p / pk  # rarefaction
        return (2.0 * ck / (g - 1.0) * (r ** ((g - 1.0) / (2.0 * g)) - 1.0),
                r ** (-(g + 1.0) / (2.0 * g)) / (dk * ck))

    ps = 0.5 * (pl + pr)
    for _ in range(100):  # Newton iteration on f_L(p) + f_R(p) + u_R - u_L = 0
        f1, d1 = fk(ps, dl, pl, cl)
        f2, d2 = fk(ps, dr, pr, cr)
        pn = max(1e-12, ps - (f1 + f2 + ur - ul) / (d1 + d2))
        done = abs(pn - ps) < 1e-15 * (pn + ps)
        ps = pn
        if done:
            break
    f1, _ = fk(ps, dl, pl, cl)
    f2, _ = fk(ps, dr, pr, cr)
    us = 0.5 * (ul + ur) + 0.5 * (f2 - f1)
    gm = (g - 1.0) / (g + 1.0)
    rho = np.empty_like(xi)
    u = np.empty_like(xi)
    p = np.empty_like(xi)
    for n, s in enumerate(xi):
        if s <= us:  # left of the contact
            if ps > pl:
                d_star = dl * (ps / pl + gm) / (gm * ps / pl + 1.0)
                sl = ul - cl * math.sqrt((g + 1.0) / (2.0 * g) * ps / pl + (g - 1.0) / (2.0 * g))
                rho[n], u[n], p[n] = (dl, ul, pl) if s < sl else (d_star, us, ps)
            else:
                d_star = dl * (ps / pl) ** (1.0 / g)
                c_star = cl * (ps / pl) ** ((g - 1.0) / (2.0 * g))
                head, tail = ul - cl, us - c_star
                if s < head:
                    rho[n], u[n], p[n] = dl, ul, pl
                elif s > tail:
                    rho[n], u[n], p[n] = d_star, us, ps
                else:
                    w = 2.0 / (g + 1.0) + gm / cl * (ul - s)
                    rho[n] = dl * w ** (2.0 / (g - 1.0))
                    u[n] = 2.0 / (g + 1.0) * (cl + (g - 1.0) / 2.0 * ul + s)
                    p[n] = pl * w ** (2.0 * g / (g - 1.0))
        else:  # right of the contact
            if ps > pr:
                d_star = dr * (ps / pr + gm) / (gm * ps / pr + 1.0)
                sr = ur + cr * math.sqrt((g + 1.0) / (2.0 * g) * ps / pr + (g - 1.0) / (2.0 * g))
                rho[n], u[n], p[n] = (dr, ur, pr) if s > sr else (d_star, us, ps)
            else:
                d_star = dr * (ps / pr) ** (1.0 / g)
                c_star = cr * (ps / pr) ** ((g - 1.0) / (2.0 * g))
                head, tail = ur + cr, us + c_star
                if s > head:
                    rho[n], u[n], p[n] = dr, ur, pr
                elif s < tail:
                    rho[n], u[n], p[n] = d_star, us, ps
                else:
                    w = 2.0 / (g + 1.0) - gm / cr * (ur - s)
                    rho[n] = dr * w ** (2.0 / (g - 1.0))
                    u[n] = 2.0 / (g + 1.0) * (-cr + (g - 1.0) / 2.0 * ur + s)
                    p[n] = pr * w ** (2.0 * g / (g - 1.0))
    return rho, u, p, ps, us


def shock_speed(left, right, g):
    """The right-moving shock's speed in Sod's problem."""
    _, _, _, ps, _ = exact_riemann(left, right, g, np.zeros(1))
    dr, ur, pr = right
    cr = math.sqrt(g * pr / dr)
    return ur + cr * math.sqrt((g + 1.0) / (2.0 * g) * ps / pr + (g - 1.0) / (2.0 * g))


def tube_deck(axis):
    """Sod's tube of N cells along `axis` on [0, 1], walls at both ends."""
    n = [NT, NT, NT]
    n[axis] = N
    dx = 1.0 / N
    ext = [(0.0, NT * dx)] * 3
    ext[axis] = (0.0, 1.0)
    bcs = [BC_PERIODIC] * 3
    bcs[axis] = BC_USER
    p = default_params(gamma=GAMMA, dt_multiplier=0.8)  # visc1 = 0.1, visc2 = 0.5
    for side, name in enumerate("xyz"):
        setattr(p, name + "bc_min", bcs[side])
        setattr(p, name + "bc_max", bcs[side])
    m = grid(n[0], n[1], n[2], ext[0], ext[1], ext[2], bcs=tuple(bcs))
    st = State.zeros(*n)
    shape = [1, 1, 1]
    shape[axis] = -1
    xc = m["xyz"[axis] + "c"].reshape(shape)
    left = xc < 0.5
    rho = np.where(left, LEFT[0], RIGHT[0])
    pres = np.where(left, LEFT[2], RIGHT[2])
    st["rho"][...] = np.broadcast_to(rho, st["rho"].shape)
    st["energy"][...] = np.broadcast_to(pres / ((GAMMA - 1.0) * rho), st["energy"].shape)
    return decks.Deck("sod_tube", p, n[0], n[1], n[2], m, st, nsteps=0)


def run_tube(s):
    """Steps until t >= T_END, as the main loop of lare3d.f90:80-89."""
    t, step = 0.0, 0
    while t < T_END and step < 2000:
        t, _ = s.step(step)
        step += 1
    return t


def tube_profile(rho, axis):
    """Density of cells 1..N along the tube, averaged across it."""
    idx = [slice(2, 2 + NT)] * 3
    idx[axis] = slice(2, 2 + N)
    others = tuple(a for a in range(3) if a != axis)
    return rho[tuple(idx)].mean(axis=others)


def tube_errors(prof, x, t):
    """(mean |rho - exact|, shock position - exact, plateau errors) of a profile."""
    exact, _, _, _, us = exact_riemann(LEFT, RIGHT, GAMMA, (x - 0.5) / t)
    l1 = float(np.mean(np.abs(prof - exact)))
    # the shock: where the density falls through the midpoint of its jump, right of the contact
    _, _, _, ps, _ = exact_riemann(LEFT, RIGHT, GAMMA, np.zeros(1))
    gm = (GAMMA - 1.0) / (GAMMA + 1.0)
    d_post = RIGHT[0] * (ps / RIGHT[2] + gm) / (gm * ps / RIGHT[2] + 1.0)
    mid = 0.5 * (d_post + RIGHT[0])
    xs_exact = 0.5 + shock_speed(LEFT, RIGHT, GAMMA) * t
    right = np.nonzero((x > 0.5 + us * t) & (prof < mid))[0]
    i = right[0]
    xs = x[i - 1] + (prof[i - 1] - mid) / (prof[i - 1] - prof[i]) * (x[i] - x[i - 1])
    # the plateau between the contact and the shock, away from both
    plateau = (x > 0.5 + us * t + 0.04) & (x < xs_exact - 0.04)
    dplat = float(np.max(np.abs(prof[plateau] - d_post)))
    return l1, xs - xs_exact, dplat


L1_BAR = 0.005       # mean |rho - exact| over the tube
SHOCK_BAR = 1.5      # cells
PLATEAU_BAR = 0.005  # max |rho - exact| on the post-shock plateau


def oracle_sim(deck):
    from oracle import oracle
    return oracle.simulation(deck)


@pytest.mark.parametrize("axis", [0, 1, 2], ids=["x", "y", "z"])
def test_sod_tube_matches_the_exact_solution(built, axis):
    d = tube_deck(axis)
    s = oracle_sim(d)
    s.start(d.state)
    t = run_tube(s)
    assert T_END <= t < T_END + 0.01
    x = d.metrics["xyz"[axis] + "c"][2:2 + N]
    l1, dxs, dplat = tube_errors(tube_profile(s.get_field("rho"), axis), x, t)
    assert l1 < L1_BAR, l1
    assert abs(dxs) < SHOCK_BAR / N, dxs * N
    assert dplat < PLATEAU_BAR, dplat


def test_sod_tube_axes_agree(built):
    prof = []
    for axis in range(3):
        d = tube_deck(axis)
        s = oracle_sim(d)
        s.start(d.state)
        run_tube(s)
        prof.append(tube_profile(s.get_field("rho"), axis))
    assert np.abs(prof[1] - prof[0]).max() <= 1e-14 and np.abs(prof[2] - prof[0]).max() <= 1e-14
